"""Builds tests/golden/tree_traces.json from the reference's d3-quadtree traces.

The reference stores 19 traces recorded from d3-quadtree 3.0.1
(test/fixtures/tree-traces.json, written by scripts/tree-traces.js): per point
set the inputs (f64 bit patterns), the extent after `cover`, the tree shape
with leaf chains, and the `visit` / `visitAfter` callback records. This script
keeps the inputs and replaces each structure by the SHA-256 of its canonical
JSON (`canonical` below), so the fixture is small and still bit-exact. The
tests rebuild the same structures from a built tree and compare digests.

    python tests/golden/make_tree_golden.py <reference checkout>/test/fixtures/tree-traces.json
"""

import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def canonical(obj):
    return hashlib.sha256(json.dumps(obj, separators=(",", ":")).encode()).hexdigest()


def main(src):
    with open(src) as f:
        traces = json.load(f)
    out = {}
    for name, t in traces.items():
        out[name] = {
            "x": t["x"],
            "y": t["y"],
            "extent": t["extent"],
            "shape": canonical(t["shape"]),
            "visit": canonical(t["visit"]),
            "after": canonical(t["after"]),
            "cells": len(t["visit"]),
        }
    dst = os.path.join(HERE, "tree_traces.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("%d traces -> %s" % (len(out), dst))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_tree_golden.py <path to the reference's test/fixtures/tree-traces.json>")
    main(sys.argv[1])
