"""find (simulation.js:157-178) as the device reduction, and custom forces
between core forces (simulation.js:66-76): GPU core == oracle core."""

import math

import numpy as np
import pytest

import helpers as H
import parity as P

pkg = H.pkg
pytestmark = pytest.mark.gpu


def _sim(core, n, seed=2):
    # links need two distinct nodes: the smallest cases have none
    nodes, src, tgt = H.scenarios.exact_graph(n, 2 * n if n > 1 else 0, 0.01, 0.01, 0.01, seed)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    if n > 1:
        sim.force("link", pkg.forceLink(src, tgt))
    return nodes, sim


@pytest.mark.parametrize("n", [1, 3, 5000, 50000])
def test_gpu_find_bitwise(ocore, gcore, n):
    na, sa = _sim(ocore, n)
    nb, sb = _sim(gcore, n)
    try:
        for ticks in (0, 3):
            if ticks:
                sa.tick(ticks)
                sb.tick(ticks)
            k = min(n - 1, 7)
            qs = [(0.0, 0.0, None), (float(na.x[k]), float(na.y[k]), None),
                  (float(na.x[k]) + 0.5, float(na.y[k]), 2.0), (1e6, 1e6, 10.0),
                  (-100.0, 250.0, math.inf), (3.0, -4.0, math.nan), (5.0, 5.0, 0.0)]
            for q in qs:
                assert sa.find(*q) == sb.find(*q), (ticks, q)
    finally:
        sa.close()
        sb.close()


def test_gpu_find_nan_and_ties(ocore, gcore):
    n = 4096
    xs = np.round(np.random.default_rng(3).uniform(-10, 10, n))
    ys = np.round(np.random.default_rng(4).uniform(-10, 10, n))
    xs[::13] = np.nan
    res = []
    for core in (ocore, gcore):
        nd = pkg.Nodes(n, x=xs, y=ys)
        sim = pkg.forceSimulation(nd, core=core)
        try:
            res.append([sim.find(float(x), float(y), r) for x, y, r in
                        [(0.0, 0.0, None), (2.0, -3.0, 1.5), (0.4, 0.6, None), (20.0, 20.0, 1.0)]])
        finally:
            sim.close()
    assert res[0] == res[1]


class _Damp:
    """A custom force: vx, vy *= 0.97 on every node."""

    def initialize(self, nodes, random):
        self.nodes = nodes
        self.r = random()

    def __call__(self, alpha):
        self.nodes.vx[:] *= 0.97
        self.nodes.vy[:] *= 0.97


def _with_custom(core):
    nodes, src, tgt = H.scenarios.exact_graph(3000, 6000, 0.01, 0.01, 0.01, 5)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.force("damp", _Damp())
    sim.force("link", pkg.forceLink(src, tgt))
    sim.force("collide", pkg.forceCollide(4))
    sim.force("center", pkg.forceCenter(0, 0))
    return nodes, sim


def test_gpu_custom_force_between_core_forces(ocore, gcore):
    P.run_pair(_with_custom, ocore, gcore, 6, step=2)
