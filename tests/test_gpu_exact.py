"""Exact mode on the B200 against the CPU oracle, bit for bit after every tick.

The oracle is pinned to d3-quadtree's traces and the reference's fast-mode
digests (test_oracle.py); here the CUDA engine must reproduce the oracle's
f64 bits (Object.is semantics: -0 and NaN payloads included) for positions,
velocities, alpha and the random stream position.
"""

import math

import numpy as np
import pytest

import helpers as H
import parity as P

pkg, sc = H.pkg, H.scenarios
pytestmark = pytest.mark.gpu

TREE_GOLDEN = H.load_tree_golden()


@pytest.mark.parametrize("name", sorted(TREE_GOLDEN))
def test_gpu_tree_matches_d3_quadtree_trace(gcore, name):
    H.check_trace(gcore, name, TREE_GOLDEN[name])


def test_gpu_tree_random_100000(ocore, gcore):
    """scripts/tree-traces.js:67-68: 100,000 points, lcg(8), compared with the oracle."""
    rnd = pkg.d3_lcg(8)
    xs, ys = np.empty(100000), np.empty(100000)
    for i in range(100000):
        xs[i] = (rnd() - 0.5) * 1e4
        ys[i] = (rnd() - 0.5) * 1e4
    a, b = H.trace(ocore, xs, ys), H.trace(gcore, xs, ys)
    assert a["extent"] == b["extent"] and a["cells"] == b["cells"]
    assert a["visit"] == b["visit"] and a["after"] == b["after"]


def _defaults(n, m, seed=1, collide=None, **kw):
    def setup(core):
        return sc.setup_exact(pkg, core, n, m, collide_radius=collide, seed=seed, **kw)
    return setup


def test_gpu_exact_1k_default_forces_300_ticks(ocore, gcore):
    """n = 1,000, m = 2,000: manyBody + link + center, every tick bitwise."""
    P.run_pair(_defaults(1000, 2000), ocore, gcore, 300)


def test_gpu_exact_collide_coincident_small(ocore, gcore):
    """Collide + coincident, near-duplicate and pinned nodes (jiggle paths)."""
    P.run_pair(_defaults(3000, 6000, collide=5, coincident=0.01, near=0.01, pinned=0.005),
               ocore, gcore, 60)


def test_gpu_exact_collide_runs_in_parallel(ocore, gcore):
    """The parallel collide path itself (not its serial fallback) matches."""
    setup = _defaults(4000, 8000, collide=5)
    na, sa = setup(ocore)
    nb, sb = setup(gcore)
    try:
        serial_ticks = 0
        for t in range(30):
            sa.tick()
            sb.tick()
            serial_ticks += int(gcore.sim_stat(sb.ctx.h, 2))
            assert P.first_difference(na, nb) is None, "tick %d" % (t + 1)
        assert serial_ticks < 30
    finally:
        sa.close()
        sb.close()


def test_gpu_exact_collide_exact_traversal_path(ocore, gcore, monkeypatch):
    """Every collide turn takes the warp-parallel exact traversal (the path a
    node pushed beyond its margin takes), bitwise with the oracle."""
    monkeypatch.setenv("D3_COLLIDE_FORCE_TRAVERSE", "1")
    P.run_pair(_defaults(4000, 8000, collide=5, coincident=0.01, near=0.01), ocore, gcore, 20)


def test_gpu_exact_d3_collide_known_answers(ocore, gcore):
    """test/d3/collide-test.js scenarios, every tick bitwise with the oracle."""
    def three(core):
        sim = pkg.forceSimulation(core=core).force("collide", pkg.forceCollide(1))
        nd = pkg.Nodes(3)
        sim.nodes(nd)
        return nd, sim
    P.run_pair(three, ocore, gcore, 10)

    def ten(core):
        nd = pkg.Nodes(10, x=[0] * 10, y=[0] * 10)
        sim = pkg.forceSimulation(core=core).nodes(nd).force("collide", pkg.forceCollide())
        return nd, sim
    P.run_pair(ten, ocore, gcore, 50)


def test_gpu_exact_forces_x_y_radial(ocore, gcore):
    def setup(core):
        nodes, sim = sc.setup_exact(pkg, core, 500, 0)
        sim.force("x", pkg.forceX(10)).force("y", pkg.forceY(-20))
        sim.force("radial", pkg.forceRadial(100, 5, 5))
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 30)


def test_gpu_host_random_source(ocore, gcore):
    """randomSource(fn): draws pulled from the caller's function in d3's order."""
    def setup(core):
        nd = pkg.Nodes(10, x=[0] * 10, y=[0] * 10)
        sim = pkg.forceSimulation(core=core).nodes(nd)
        sim.force("charge", pkg.forceManyBody()).force("collide", pkg.forceCollide())
        sim.randomSource(pkg.d3_lcg(12345))
        return nd, sim
    P.run_pair(setup, ocore, gcore, 20)


@pytest.mark.slow
def test_gpu_exact_50k_collide(ocore, gcore):
    """The 50k + collide benchmark workload, bitwise for the first ticks."""
    P.run_pair(_defaults(50000, 100000, collide=5, coincident=0.01, near=0.01, pinned=0.005),
               ocore, gcore, 5)


def test_gpu_sim_tick_path_matches(ocore, gcore):
    """sim_tick (device-resident ticks, center sums overlapped on a side
    stream) gives the same bits as one force_run per force per tick."""
    setup = _defaults(5000, 10000, collide=5, coincident=0.01, near=0.01, pinned=0.005)
    na, sa = setup(ocore)
    nb, sb = setup(gcore)
    try:
        for chunk in (1, 4, 15):
            sa.tick(chunk)
            sb.run(chunk)
            assert P.first_difference(na, nb) is None, "after a run of %d" % chunk
            assert sa.alpha() == sb.alpha()
        assert ocore.sim_get_lcg(sa.ctx.h) == gcore.sim_get_lcg(sb.ctx.h)
    finally:
        sa.close()
        sb.close()


def test_gpu_force_run_per_force_path_matches(ocore, gcore):
    """tick() driven the reference facade's way, one force_run per force per
    tick (no sim_tick), with the device LCG: bitwise with the oracle."""
    base = _defaults(3000, 6000, collide=5, coincident=0.01, near=0.01, pinned=0.005)

    def setup(core):
        nodes, sim = base(core)
        sim.engine_ticks = False
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 30)


def test_gpu_bounded_wait_reports_failure_and_recovers(gcore):
    """A device wait that nothing completes gives up after its budget: the call
    returns D3_WORKER_FAILED (-4) and the simulation keeps working (the status
    is reported once, then clear)."""
    nodes, sim = sc.setup_exact(pkg, gcore, 2000, 4000, collide_radius=3)
    try:
        h = sim.ctx.h
        assert gcore.sim_selftest_wait(h, 2000) == -4
        assert gcore.sim_sync_out(h) == 0
        sim.tick(3)
        assert gcore.sim_sync_out(h) == 0
        assert all(map(lambda v: v == v, nodes.x[:10]))
    finally:
        sim.close()
