"""The facade's find and custom forces (simulation.js:49-89, 107-110,
157-178) on the oracle core: no GPU needed."""

import math

import numpy as np
import pytest

import helpers as H

pkg = H.pkg


def _find_serial(xs, ys, x, y, radius=None):
    """simulation.js:157-178, statement by statement."""
    r2 = math.inf if radius is None else radius * radius
    closest = None
    for i in range(len(xs)):
        dx, dy = x - float(xs[i]), y - float(ys[i])
        d2 = dx * dx + dy * dy
        if d2 < r2:
            closest, r2 = i, d2
    return closest


def _find_nodes(n, seed):
    rng = np.random.default_rng(seed)
    xs = np.round(rng.uniform(-50, 50, n), 1)  # rounded: many equal distances
    ys = np.round(rng.uniform(-50, 50, n), 1)
    xs[::97] = np.nan
    ys[5::89] = np.nan
    if n > 10:
        xs[7], ys[7] = xs[3], ys[3]  # an exact duplicate after a lower index
    return xs, ys


QUERIES = [(0.0, 0.0, None), (12.3, -4.5, None), (12.3, -4.5, 3.0), (100.0, 100.0, 1.0),
           (0.05, 0.05, 0.0), (-7.0, 7.0, -2.5), (1.0, 1.0, math.nan), (math.nan, 0.0, None),
           (1e300, 1e300, None), (-20.0, 30.0, math.inf)]


@pytest.mark.parametrize("n", [0, 1, 2, 1000])
def test_find_matches_the_serial_scan(ocore, n):
    xs, ys = _find_nodes(n, n)
    nd = pkg.Nodes(n, x=xs, y=ys)
    sim = pkg.forceSimulation(nd, core=ocore)
    try:
        for q in QUERIES + [(xs[3], ys[3], None)] if n > 10 else QUERIES:
            assert sim.find(*q) == _find_serial(nd.x, nd.y, *q), q
    finally:
        sim.close()


class _Kick:
    """A custom force: vx += 1 on every node, recording the alphas it gets."""

    def __init__(self):
        self.alphas = []
        self.nodes = None
        self.draws = []

    def initialize(self, nodes, random):
        self.nodes = nodes
        self.draws = [random(), random()]

    def __call__(self, alpha):
        self.alphas.append(alpha)
        self.nodes.vx[:] += 1.0


def test_custom_force_sees_and_changes_the_node_table(ocore):
    nd = pkg.Nodes(3, x=[0.0, 10.0, 20.0], y=[0.0, 0.0, 5.0], vx=[0.0] * 3, vy=[0.0] * 3)
    sim = pkg.forceSimulation(nd, core=ocore)
    try:
        kick = _Kick()
        sim.force("kick", kick)
        sim.tick()
        # integrate: vx = (0 + 1) * 0.6, x += vx
        assert list(nd.vx) == [0.6, 0.6, 0.6]
        assert list(nd.x) == [0.6, 10.6, 20.6]
        assert list(nd.y) == [0.0, 0.0, 5.0]
        a1 = 1 + (0 - 1) * (1 - math.pow(0.001, 1 / 300))
        assert kick.alphas == [a1]
        sim.tick(2)
        assert len(kick.alphas) == 3 and kick.alphas[0] > kick.alphas[1] > kick.alphas[2]
    finally:
        sim.close()


def test_custom_force_draws_from_the_shared_stream(ocore):
    """initialize(nodes, random) draws from d3's LCG, whose state the core
    keeps for its own jiggles (one stream per simulation)."""
    nd = pkg.Nodes(2, x=[0.0, 1.0], y=[0.0, 1.0])
    sim = pkg.forceSimulation(nd, core=ocore)
    try:
        ref = pkg.d3_lcg(1)
        kick = _Kick()
        sim.force("kick", kick)
        assert kick.draws == [ref(), ref()]
        nxt = (1664525 * ocore.sim_get_lcg(sim.ctx.h) + 1013904223) % 4294967296
        assert nxt / 4294967296 == ref()
    finally:
        sim.close()


def _graph(core, custom):
    nodes, src, tgt = H.scenarios.exact_graph(400, 800, 0.01, 0.01, 0.01, 3)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    if custom is not None:
        sim.force("custom", custom)
    sim.force("link", pkg.forceLink(src, tgt))
    sim.force("collide", pkg.forceCollide(4))
    sim.force("center", pkg.forceCenter(0, 0))
    return nodes, sim


def test_identity_custom_force_changes_nothing(ocore):
    """A custom force that does nothing: the copy-out / copy-in around it
    leaves the ticks bit-identical to the run without it."""
    na, sa = _graph(ocore, None)
    nb, sb = _graph(ocore, lambda alpha: None)
    try:
        sa.tick(5)
        sb.tick(5)
        for f in ("x", "y", "vx", "vy"):
            assert np.array_equal(np.asarray(getattr(na, f)).view(np.uint64),
                                  np.asarray(getattr(nb, f)).view(np.uint64)), f
        assert sa.alpha() == sb.alpha()
    finally:
        sa.close()
        sb.close()


def test_engine_path_refuses_a_custom_force(ocore):
    nodes, sim = _graph(ocore, lambda alpha: None)
    try:
        with pytest.raises(ValueError):
            sim.device_begin()
        sim.run(2)  # run() falls back to tick() with a custom force
    finally:
        sim.close()


def test_fixed_bits_from_fx_fy(ocore):
    """sim_set_fixed_source(h, 1): each upload derives src/core.js:130's bits
    from fx / fy (NaN = not set); mode 0 keeps the array as written."""
    C = H.C
    h = ocore.sim_create()
    try:
        assert ocore.sim_set_node_count(h, 4) >= 0
        fx = ocore.f64_view(ocore.sim_ptr(h, C.PTR_FX), 4)
        fy = ocore.f64_view(ocore.sim_ptr(h, C.PTR_FY), 4)
        fixed = ocore.u8_view(ocore.sim_ptr(h, C.PTR_FIXED), 4)
        fx[:] = [np.nan, 1.0, np.nan, -0.0]
        fy[:] = [np.nan, np.nan, 2.0, np.inf]
        fixed[:] = 7
        assert ocore.sim_sync_in(h) == 0
        assert list(fixed) == [7, 7, 7, 7]
        assert ocore.sim_set_fixed_source(h, 2) == C.BAD_ARGUMENT
        assert ocore.sim_set_fixed_source(h, 1) == 0
        assert ocore.sim_sync_in(h) == 0
        assert list(fixed) == [0, 1, 2, 3]
    finally:
        ocore.sim_destroy(h)


def test_nodes_reinitializes_custom_forces(ocore):
    """simulation.js:125-127: nodes(_) re-runs every force's initialize with
    the new table (a custom force's initialize(nodes, random) included)."""
    nd = pkg.Nodes(2, x=[0.0, 1.0], y=[0.0, 1.0])
    sim = pkg.forceSimulation(nd, core=ocore)
    try:
        kick = _Kick()
        sim.force("kick", kick)
        assert kick.nodes is nd
        nd2 = pkg.Nodes(5)
        sim.nodes(nd2)
        assert kick.nodes is nd2 and len(kick.draws) == 2
        sim.tick()
        assert np.all(np.asarray(nd2.vx) == 0.6)
    finally:
        sim.close()


def _linked(core, by_id):
    n = 60
    nodes = pkg.Nodes(n)
    rng = np.random.default_rng(9)
    src = rng.integers(0, n, 120)
    tgt = (src + 1 + rng.integers(0, n - 1, 120)) % n
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    if by_id:
        link = pkg.forceLink(["n%d" % v for v in src], ["n%d" % v for v in tgt])
        link.id(lambda i: "n%d" % i)
    else:
        link = pkg.forceLink(src, tgt)
    sim.force("link", link)
    return nodes, sim, link, src, tgt


def test_link_ids_resolve_like_indices(ocore):
    """link.js:41-50: endpoints given as node ids through id() give the same
    links, counts, bias and ticks as the same links given as indices."""
    na, sa, la, src, tgt = _linked(ocore, False)
    nb, sb, lb, _, _ = _linked(ocore, True)
    try:
        assert np.array_equal(lb.links()[0], src) and np.array_equal(lb.links()[1], tgt)
        assert np.array_equal(la.bias, lb.bias) and np.array_equal(la.count, lb.count)
        sa.tick(4)
        sb.tick(4)
        for f in ("x", "y", "vx", "vy"):
            assert np.array_equal(np.asarray(getattr(na, f)).view(np.uint64),
                                  np.asarray(getattr(nb, f)).view(np.uint64)), f
    finally:
        sa.close()
        sb.close()


def test_link_unknown_id_and_new_links(ocore):
    nd = pkg.Nodes(3)
    sim = pkg.forceSimulation(nd, core=ocore)
    try:
        link = pkg.forceLink(["a"], ["zz"]).id(lambda i: "abc"[i])
        with pytest.raises(KeyError):
            sim.force("link", link)
        link = pkg.forceLink([0], [1])
        sim.force("link", link)
        assert list(link.count) == [1, 1, 0]
        link.links([0, 2, 2], [1, 1, 0])  # initializes again
        assert list(link.count) == [2, 2, 2]
        assert list(link.links()[0]) == [0, 2, 2]
    finally:
        sim.close()


def test_threads_is_accepted(ocore):
    sim = pkg.forceSimulation(pkg.Nodes(2), core=ocore)
    try:
        assert sim.threads(4) is sim and sim.threads(None) is sim
        assert sim.threads(float("nan")) is sim and sim.threads() == 0
    finally:
        sim.close()


def _bits(nd):
    return [np.asarray(getattr(nd, f)).view(np.uint64).copy() for f in ("x", "y", "vx", "vy")]


def _run(core, make, n=40, ticks=3):
    nd = pkg.Nodes(n)
    sim = pkg.forceSimulation(nd, core=core)
    try:
        for name, f in make():
            sim.force(name, f)
        sim.tick(ticks)
        return _bits(nd)
    finally:
        sim.close()


def test_force_getters_return_what_was_set():
    mb = pkg.forceManyBody().strength(-12).distanceMin(2).distanceMax(50).theta(0.5)
    assert mb.strength()(3) == -12 and mb.distanceMin() == 2 and mb.distanceMax() == 50
    assert mb.theta() == 0.5
    co = pkg.forceCollide().radius(3).strength(0.7).iterations(2)
    assert co.radius()(0) == 3 and co.strength() == 0.7 and co.iterations() == 2
    ce = pkg.forceCenter().x(3).y(-1).strength(0.5)
    assert (ce.x(), ce.y(), ce.strength()) == (3, -1, 0.5)
    fx, fy = pkg.forceX().x(10).strength(0.5), pkg.forceY().y(-4)
    assert fx.x()(0) == 10 and fx.strength()(0) == 0.5 and fy.y()(1) == -4
    ra = pkg.forceRadial(5).strength(0.2).x(1).y(2).radius(7)
    assert ra.radius()(0) == 7 and ra.strength()(0) == 0.2 and (ra.x(), ra.y()) == (1, 2)
    li = pkg.forceLink([0, 0, 1], [1, 2, 2]).iterations(3).distance(12)
    assert li.iterations() == 3 and li.distance()(0) == 12


def test_default_link_strength_getter(ocore):
    sim = pkg.forceSimulation(pkg.Nodes(3), core=ocore)
    try:
        li = pkg.forceLink([0, 0], [1, 2])
        sim.force("link", li)
        assert li.strength()(0) == 1.0 / min(2, 1)  # link.js:30-32
    finally:
        sim.close()


def test_setters_equal_constructor_arguments(ocore):
    """radial / center / x / y configured by setters tick bit for bit like
    the same values given to the constructors."""
    a = _run(ocore, lambda: [("r", pkg.forceRadial(7, 1, 2).strength(0.2)),
                             ("c", pkg.forceCenter(3, -1).strength(0.5)),
                             ("x", pkg.forceX(10).strength(0.3)), ("y", pkg.forceY(-4))])
    b = _run(ocore, lambda: [("r", pkg.forceRadial(5).strength(0.2).x(1).y(2).radius(7)),
                             ("c", pkg.forceCenter().x(3).y(-1).strength(0.5)),
                             ("x", pkg.forceX().x(10).strength(0.3)), ("y", pkg.forceY().y(-4))])
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_force_x_known_answer(ocore):
    """simple.zig:51-62 then integrate: vx += (target - x) strength alpha;
    vx *= 0.6; x += vx."""
    nd = pkg.Nodes(1, x=[2.0], y=[0.0], vx=[0.0], vy=[0.0])
    sim = pkg.forceSimulation(nd, core=ocore).force("x", pkg.forceX().x(10).strength(0.5))
    try:
        sim.tick()
        a = 1 + (0 - 1) * (1 - math.pow(0.001, 1 / 300))
        vx = (0.0 + (10 - 2.0) * 0.5 * a) * 0.6
        assert nd.vx[0] == vx and nd.x[0] == 2.0 + vx
    finally:
        sim.close()
