"""Shared test helpers: package import, cores, d3-quadtree trace rebuild."""

import hashlib
import importlib
import json
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

pkg = importlib.import_module("d3-force-wasm_b200")
scenarios = importlib.import_module("d3-force-wasm_b200.scenarios")
C = pkg.core
import oracle  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
NONE = 0xFFFFFFFF


def oracle_core():
    return oracle.load(pkg)


def bits(v):
    return struct.pack("<d", float(v)).hex() if False else "%016x" % struct.unpack("<Q", struct.pack("<d", float(v)))[0]


def unbits(s):
    return struct.unpack("<d", struct.pack("<Q", int(s, 16)))[0]


def canonical(obj):
    return hashlib.sha256(json.dumps(obj, separators=(",", ":")).encode()).hexdigest()


def build_tree(core, xs, ys):
    """Loads positions into a fresh simulation of `core` and builds the tree."""
    h = core.sim_create()
    n = len(xs)
    assert core.sim_set_node_count(h, n) >= 0
    if n:
        core.f64_view(core.sim_ptr(h, C.PTR_X), n)[:] = xs
        core.f64_view(core.sim_ptr(h, C.PTR_Y), n)[:] = ys
        core.f64_view(core.sim_ptr(h, C.PTR_VX), n)[:] = 0
        core.f64_view(core.sim_ptr(h, C.PTR_VY), n)[:] = 0
    assert core.sim_sync_in(h) == 0
    assert core.tree_build(h, 0) >= 0
    return h


def trace(core, xs, ys):
    """The d3-quadtree trace (scripts/tree-traces.js:84-101 format) of the
    tree `core` builds for the points."""
    h = build_tree(core, xs, ys)
    t = core.tree(h)
    cells, perm = t["cells"], t["perm"]
    n_cells = len(cells)
    visit = core.order(h, 0) if n_cells else []
    after = core.order(h, 1) if n_cells else []
    core.sim_destroy(h)

    def is_leaf(c):
        return all(int(k) == NONE for k in cells[c]["child"])

    def chain(c):
        f, k = int(cells[c]["first"]), int(cells[c]["count"])
        return [int(perm[i]) for i in range(f + k - 1, f - 1, -1)]

    def shape(c):
        if c == NONE:
            return None
        if is_leaf(c):
            return {"l": chain(c)}
        return [shape(int(k)) for k in cells[c]["child"]]

    def rec(c):
        cc = cells[c]
        return [chain(c)[0] if is_leaf(c) else -1, bits(cc["x0"]), bits(cc["y0"]), bits(cc["x1"]),
                bits(cc["y1"])]

    sys.setrecursionlimit(100000)
    return {
        "extent": [bits(v) for v in t["extent"]],
        "shape": shape(int(t["root"])) if n_cells else None,
        "visit": [rec(int(c)) for c in visit],
        "after": [rec(int(c)) for c in after],
        "cells": n_cells,
    }


def load_tree_golden():
    with open(os.path.join(GOLDEN, "tree_traces.json")) as f:
        return json.load(f)


def check_trace(core, name, ref):
    xs = np.array([unbits(s) for s in ref["x"]])
    ys = np.array([unbits(s) for s in ref["y"]])
    got = trace(core, xs, ys)
    assert got["extent"] == ref["extent"], "%s: extent" % name
    assert got["cells"] == ref["cells"], "%s: cell count %d vs %d" % (name, got["cells"], ref["cells"])
    assert canonical(got["shape"]) == ref["shape"], "%s: shape and leaf chains" % name
    assert canonical(got["visit"]) == ref["visit"], "%s: visit order and bounds" % name
    assert canonical(got["after"]) == ref["after"], "%s: visitAfter order and bounds" % name


def clustered_pairs(n, seed, scale=2.0 ** -20):
    """n points: n/2 uniform in [-400, 400)^2, each with a partner offset by
    between 0.5 and 1 x 800 * scale on each axis. d3's quadtree separates a
    pair only at the level where the two fall in different quadrants, so each
    pair hangs a chain of single-child cells below the uniform points' levels:
    at scale 2^-20 the tree needs more than the 4n + 1024 cells the engine
    reserves."""
    rng = np.random.default_rng(seed)
    b = n // 2
    x = np.empty(n)
    y = np.empty(n)
    x[:b] = (rng.random(b) - 0.5) * 800
    y[:b] = (rng.random(b) - 0.5) * 800
    off = 800 * scale * (0.5 + 0.5 * rng.random((b, 2)))
    x[b:2 * b] = x[:b] + off[:, 0]
    y[b:2 * b] = y[:b] + off[:, 1]
    if n % 2:
        x[-1] = y[-1] = 0.0
    return x, y
