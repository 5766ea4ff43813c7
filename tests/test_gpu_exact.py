"""Exact mode on the B200 against the CPU oracle, bit for bit after every tick.

The oracle is pinned to d3-quadtree's traces and the reference's fast-mode
digests (test_oracle.py); here the CUDA engine must reproduce the oracle's
f64 bits (Object.is semantics: -0 and NaN payloads included) for positions,
velocities, alpha and the random stream position.
"""

import math
import os

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
def test_gpu_exact_50k_collide_every_tick_of_300(ocore, gcore):
    """The 50k + collide benchmark workload (1% coincident, 1% offsets below
    1e-12, 0.5% pinned), bitwise with the oracle after every one of its 300
    ticks: positions, velocities, alpha, and the random stream position at
    ticks 1, 5, 25, 100, 200 and 300 (test/parity/parity-test.js:23-58 checks
    each tick with Object.is and the stream's next value at the end). The
    oracle runs on all host threads; its threaded ticks are the serial ones
    bit for bit (test_oracle.py, test_threaded_oracle_ticks_bitwise)."""
    setup = _defaults(50000, 100000, collide=5, coincident=0.01, near=0.01, pinned=0.005)
    na, sa = setup(ocore)
    nb, sb = setup(gcore)
    ocore.lib.oracle_set_threads(sa.ctx.h, os.cpu_count() or 1)
    try:
        assert P.first_difference(na, nb) is None, "after initialize"
        for t in range(1, 301):
            sa.tick()
            sb.tick()
            d = P.first_difference(na, nb)
            assert d is None, "tick %d: %s" % (t, d)
            assert sa.alpha() == sb.alpha(), "tick %d: alpha" % t
            if t in (1, 5, 25, 100, 200, 300):
                assert ocore.sim_get_lcg(sa.ctx.h) == gcore.sim_get_lcg(sb.ctx.h), \
                    "tick %d: random stream position" % t
    finally:
        sa.close()
        sb.close()


def test_gpu_tree_overflow_leaves_an_empty_tree(ocore, gcore):
    """A tree that needs more cells than the engine reserves (4n + 1024; the
    clustered pairs below need about 7.8n, test_oracle.py checks that on the
    oracle) is reported, not written past its buffers: tree_build returns
    D3_WORKER_FAILED with an empty tree, a many-body force_run leaves the
    velocities as they were and the next sync reports the failure once, and
    the simulation then works normally on points that fit."""
    n = 2000
    x, y = H.clustered_pairs(n, 3)
    h = gcore.sim_create()
    try:
        assert gcore.sim_set_node_count(h, n) >= 0
        gcore.sim_set_sync(h, H.C.SYNC_EXPLICIT)
        vx0 = np.linspace(-1, 1, n)
        for w, arr in ((H.C.PTR_X, x), (H.C.PTR_Y, y), (H.C.PTR_VX, vx0), (H.C.PTR_VY, -vx0)):
            gcore.f64_view(gcore.sim_ptr(h, w), n)[:] = arr
        gcore.u8_view(gcore.sim_ptr(h, H.C.PTR_FIXED), n)[:] = 0
        assert gcore.sim_sync_in(h) == 0
        assert gcore.tree_build(h, 0) == H.C.WORKER_FAILED
        assert gcore.tree_info(h, 0) == 0
        fh = gcore.force_create(h, H.C.MANY_BODY)
        gcore.f64_view(gcore.force_ptr(h, fh, H.C.F0), n)[:] = -30.0
        gcore.force_set_scalar(h, fh, H.C.THETA2, 0.81)
        gcore.force_set_scalar(h, fh, H.C.DISTANCE_MIN2, 1.0)
        gcore.force_set_scalar(h, fh, H.C.DISTANCE_MAX2, float("inf"))
        assert gcore.force_run(h, fh, 1.0) == 0
        assert gcore.sim_sync_out(h) == H.C.WORKER_FAILED
        got = gcore.f64_view(gcore.sim_ptr(h, H.C.PTR_VX), n)
        assert np.array_equal(P.bits(got), P.bits(vx0))
        assert gcore.sim_sync_out(h) == 0  # reported once
        # the same nodes spread out: the tree fits and matches the oracle's
        xs, ys = H.clustered_pairs(n, 3, scale=2.0 ** -6)
        a, b = H.trace(ocore, xs, ys), H.trace(gcore, xs, ys)
        assert a["cells"] == b["cells"] and a["visit"] == b["visit"]
    finally:
        gcore.sim_destroy(h)


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
