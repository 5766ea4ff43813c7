"""Fast mode on the B200: the Jacobi link and the grid collide are per-node
passes with the reference's per-node operation order, so they match the
oracle bit for bit; the FMM is checked by RMS error."""

import numpy as np
import pytest

import helpers as H
import parity as P

pkg, sc = H.pkg, H.scenarios
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["uniform 4000", "grid 2500 with exact zero deltas"])
def test_gpu_fast_link_collide_center_bitwise(ocore, gcore, name):
    def setup(core):
        nodes, src, tgt = sc.fast_scenario(name)
        sim = pkg.forceSimulation(nodes, core=core)
        sim.force("link", pkg.forceLink(src, tgt))
        sim.force("collide", pkg.forceCollide(3))
        sim.force("center", pkg.forceCenter())
        sim.precision("fast")
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 100)


def _golden():
    import json
    import os
    with open(os.path.join(H.GOLDEN, "fast_golden.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", sc.FAST_SCENARIOS)
def test_gpu_fast_mode_matches_golden_digests(gcore, name):
    """The whole fast tick on the GPU (FMM many-body, Jacobi link, grid
    collide, center) against the reference's SHA-256 digests
    (test/fixtures/fast-golden.json) at ticks 1, 10, 100 and 300."""
    golden = _golden()[name]
    nodes, sim = sc.setup_fast_scenario(pkg, gcore, name)
    try:
        for t in range(1, sc.CHECKPOINTS[-1] + 1):
            sim.tick()
            if t in sc.CHECKPOINTS:
                assert sc.digest(nodes) == golden[str(t)], "tick %d" % t
    finally:
        sim.close()


@pytest.mark.parametrize("order,opening,dmax", [(8, 1.5, None), (4, 1.2, None), (12, 2.0, None),
                                                 (8, 1.5, 200.0), (1, 1.01, None)])
def test_gpu_fmm_bitwise_vs_oracle(ocore, gcore, order, opening, dmax):
    """FMM many-body alone, every tick bit-identical to the oracle, over
    orders, openings and a finite distanceMax (the ring test of fmm.zig:417-425)."""
    def setup(core):
        nodes, src, tgt = sc.fast_scenario("three clusters 6000")
        sim = pkg.forceSimulation(nodes, core=core)
        mb = pkg.forceManyBody()
        if dmax is not None:
            mb.distanceMax(dmax)
        sim.force("charge", mb)
        sim.precision("fast", order=order, opening=opening)
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 12)


def test_gpu_fmm_coincident_and_nan_nodes(ocore, gcore):
    """Coincident points (hashed jiggle in P2P, deep leaves past 32 points at
    depth 16) and nodes with a NaN coordinate (left out of the tree)."""
    def setup(core):
        rnd = sc.generator(7)
        n = 5000
        xs = [rnd() * 500 for _ in range(n)]
        ys = [rnd() * 500 for _ in range(n)]
        for k in range(0, 400):  # 41 points at each of 10 positions
            xs[4000 + k] = xs[k % 10]
            ys[4000 + k] = ys[k % 10]
        nodes = pkg.Nodes(n, x=xs, y=ys)
        sim = pkg.forceSimulation(nodes, core=core)
        sim.force("charge", pkg.forceManyBody())
        sim.precision("fast")
        nodes.x[17] = float("nan")  # after d3's placement of NaN positions
        nodes.y[4999] = float("nan")
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 5)
