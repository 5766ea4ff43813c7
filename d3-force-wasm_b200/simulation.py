"""d3-force's simulation and force API over the engine's C ABI.

A Python restatement of d3-force-wasm's facade: ``src/simulation.js`` (alpha
schedule, force order, tick loop, phyllotaxis start), ``src/core.js``
(`Context` copy-in / copy-out, `Slot` binding, the fast-mode SEED draw) and the
force facades ``src/{manyBody,link,collide,center,x,y,radial}.js`` (accessor
evaluation into the core's arrays). Names, defaults and arithmetic follow those
files; nodes are a `Nodes` structure of f64 arrays instead of JS objects, with
NaN standing for a missing (null / undefined) field.
"""

import ctypes
import math

import numpy as np

from . import core as C

_GET = object()  # a method called with no argument reads the value (d3's getters)

INITIAL_RADIUS = 10.0
INITIAL_ANGLE = math.pi * (3 - math.sqrt(5))  # simulation.js:14-15


class Nodes:
    """Node table: x, y, vx, vy, fx, fy as f64[n]; NaN = field not set."""

    def __init__(self, n=0, x=None, y=None, vx=None, vy=None, fx=None, fy=None):
        self.n = n
        nan = lambda: np.full(n, np.nan)  # noqa: E731
        self.x = np.array(x, np.float64) if x is not None else nan()
        self.y = np.array(y, np.float64) if y is not None else nan()
        self.vx = np.array(vx, np.float64) if vx is not None else nan()
        self.vy = np.array(vy, np.float64) if vy is not None else nan()
        self.fx = np.array(fx, np.float64) if fx is not None else nan()
        self.fy = np.array(fy, np.float64) if fy is not None else nan()

    def __len__(self):
        return self.n

    def fixed_bits(self):
        """src/core.js:130: (fx != null) | (fy != null) << 1."""
        return ((~np.isnan(self.fx)).astype(np.uint8) | ((~np.isnan(self.fy)).astype(np.uint8) << 1))


def _constant(v):
    return lambda *_: v


def _accessor(v):
    return v if callable(v) else _constant(float(v))


class Context:
    """src/core.js:89-164: one simulation handle in the core per node table."""

    def __init__(self, core):
        self.core = core
        self.h = core.sim_create()
        if not self.h:
            raise C.CoreError(C.OUT_OF_MEMORY)
        self.n = 0
        C.check(core.sim_set_sync(self.h, C.SYNC_EXPLICIT))
        # src/core.js:130's fixed bits, (fx set) | (fy set) << 1, are derived
        # from fx / fy (NaN = not set) by the engine at each upload
        C.check(core.sim_set_fixed_source(self.h, 1))
        self.live = False
        self._nodes = None  # the node table whose arrays are the mirrors
        self._views = ()
        self.precision = None  # None = exact; {"order", "opening"} = fast
        self.host_random = None  # callback for randomSource(); None = device LCG
        self._cb = None

    FIELDS = (("x", C.PTR_X), ("y", C.PTR_Y), ("vx", C.PTR_VX), ("vy", C.PTR_VY),
              ("fx", C.PTR_FX), ("fy", C.PTR_FY))

    def resize(self, n):
        if n != self.n:
            self.detach()  # the mirrors move
            C.check(self.core.sim_set_node_count(self.h, n))
            self.n = n

    def view(self, which, n):
        return self.core.f64_view(self.core.sim_ptr(self.h, which), n)

    def _bound(self, nodes):
        """True if nodes' arrays are this context's mirrors."""
        if self._nodes is not nodes or not self.n:
            return False
        return all(getattr(nodes, f) is v for (f, _), v in zip(self.FIELDS, self._views))

    def detach(self):
        """Gives the bound node table its own copies of the mirrors."""
        nodes, self._nodes, views, self._views = self._nodes, None, self._views, ()
        if nodes is not None:
            for (f, _), v in zip(self.FIELDS, views):
                if getattr(nodes, f) is v:
                    setattr(nodes, f, np.array(v, np.float64))

    def bind(self, nodes):
        """src/core.js:121-131 on the host: the node table's x, y, vx, vy,
        fx, fy become views of the pinned mirrors the first time (as the
        reference's facade views wasm memory), so later ticks copy nothing on
        the host; the fixed bits (src/core.js:130) are derived from fx / fy on
        the device."""
        n = len(nodes)
        self.resize(n)
        if n and not self._bound(nodes):
            self.detach()
            views = []
            for f, w in self.FIELDS:
                v = self.view(w, n)
                v[:] = getattr(nodes, f)
                setattr(nodes, f, v)
                views.append(v)
            self._nodes, self._views = nodes, tuple(views)

    def copy_in(self, nodes):
        """bind(), then one host-to-device sync."""
        self.bind(nodes)
        C.check(self.core.sim_sync_in(self.h))

    def copy_out(self, nodes):
        """src/core.js:133-141, after one device-to-host sync (a bound node
        table already holds the result)."""
        C.check(self.core.sim_sync_out(self.h))
        self.read_back(nodes)

    def read_back(self, nodes):
        """The mirrors' x, y, vx, vy into a node table that is not bound to
        them (a bound one already holds them)."""
        n = self.n
        if n and not self._bound(nodes):
            nodes.x[:] = self.view(C.PTR_X, n)
            nodes.y[:] = self.view(C.PTR_Y, n)
            nodes.vx[:] = self.view(C.PTR_VX, n)
            nodes.vy[:] = self.view(C.PTR_VY, n)

    def set_random(self, fn):
        """None: the device LCG; else a Python callable drawn in d3's order."""
        if fn is None:
            self._cb = None
            self.host_random = None
            return
        self._cb = C.RANDOM_FN(lambda _ctx: float(fn()))
        self.host_random = fn
        C.check(self.core.sim_set_random(self.h, self._cb, None))

    def close(self):
        if self.h:
            self.detach()
            self.core.sim_destroy(self.h)
            self.h = 0


class Slot:
    """src/core.js:174-232: a native force's handle in the core."""

    def __init__(self, kind):
        self.kind = kind
        self.ctx = None
        self.fh = 0
        self.m = 0
        self._sent = {}  # scalar slot -> the value last set (as float.hex())

    def bind(self, ctx, n):
        if ctx is not self.ctx:
            if self.ctx is not None:
                self.ctx.core.force_destroy(self.ctx.h, self.fh)
            self.fh = ctx.core.force_create(ctx.h, self.kind)
            if not self.fh:
                raise C.CoreError(C.OUT_OF_MEMORY)
            self.ctx = ctx
            self.m = 0
            self._sent = {}
        ctx.resize(n)

    def count(self, m):
        C.check(self.ctx.core.force_set_count(self.ctx.h, self.fh, m))
        self.m = m

    def f64(self, which, m):
        return self.ctx.core.f64_view(self.ctx.core.force_ptr(self.ctx.h, self.fh, which), m)

    def u32(self, which, m):
        return self.ctx.core.u32_view(self.ctx.core.force_ptr(self.ctx.h, self.fh, which), m)

    def scalar(self, which, v):
        """force_set_scalar, skipped when the slot already holds this value
        (scalars change only through this call; SEED is always sent)."""
        v = float(v)
        key = v.hex()
        if which != C.SEED and self._sent.get(which) == key:
            return
        C.check(self.ctx.core.force_set_scalar(self.ctx.h, self.fh, which, v))
        self._sent[which] = key

    def run(self, alpha, random=None):
        """src/core.js:213-231: PRECISION, fast-mode ORDER / OPENING and SEED."""
        ctx = self.ctx
        fast = ctx.precision
        self.scalar(C.PRECISION, fast["form"] if fast else 0)
        if fast:
            self.scalar(C.ORDER, fast["order"])
            self.scalar(C.OPENING, fast["opening"])
            # With the device LCG the core draws SEED itself at force_run.
            if ctx.host_random is not None and self.kind in (C.MANY_BODY, C.LINK, C.COLLIDE):
                self.scalar(C.SEED, ctx.host_random())
        C.check(ctx.core.force_run(ctx.h, self.fh, alpha))


# Bumped by every attribute a core force's methods set (its scalars, its
# nodes): Simulation.tick pushes the forces' scalars only when it moved.
_FORCE_GEN = [0]


class Force:
    kind = None

    def __setattr__(self, name, value):
        object.__setattr__(self, name, value)
        _FORCE_GEN[0] += 1

    def __init__(self):
        self.slot = Slot(self.kind)
        self.nodes = None
        self.ctx = None

    def initialize(self, nodes, ctx):
        self.nodes = nodes
        self.ctx = ctx
        self._initialize()

    def _initialize(self):
        self.slot.bind(self.ctx, len(self.nodes))

    def __call__(self, alpha):
        self._push()
        self.slot.run(alpha)

    def _push(self):
        pass


class ForceManyBody(Force):
    """src/manyBody.js: strength -30, distanceMin 1, distanceMax inf, theta 0.9."""

    kind = C.MANY_BODY

    def __init__(self):
        super().__init__()
        self._strength = _constant(-30.0)
        self.distance_min2 = 1.0
        self.distance_max2 = math.inf
        self.theta2 = 0.81

    def _initialize(self):
        n = len(self.nodes)
        self.slot.bind(self.ctx, n)
        self.slot.count(n)
        a = self.slot.f64(C.F0, n)
        for i in range(n):
            a[i] = float(self._strength(i))

    def _push(self):
        self.slot.scalar(C.THETA2, self.theta2)
        self.slot.scalar(C.DISTANCE_MIN2, self.distance_min2)
        self.slot.scalar(C.DISTANCE_MAX2, self.distance_max2)

    def strength(self, s=_GET):
        """manyBody.js:37-39"""
        if s is _GET:
            return self._strength
        self._strength = _accessor(s)
        if self.nodes is not None:
            self._initialize()
        return self

    def distanceMin(self, d=_GET):
        """manyBody.js:41-43"""
        if d is _GET:
            return math.sqrt(self.distance_min2)
        self.distance_min2 = d * d
        return self

    def distanceMax(self, d=_GET):
        """manyBody.js:45-47"""
        if d is _GET:
            return math.sqrt(self.distance_max2)
        self.distance_max2 = d * d
        return self

    def theta(self, t=_GET):
        """manyBody.js:49-51"""
        if t is _GET:
            return math.sqrt(self.theta2)
        self.theta2 = t * t
        return self


class ForceLink(Force):
    """src/link.js: links as (source, target) sequences, node indices by
    default or node ids once id() is set; degree count, bias, default
    strength 1 / min(count[source], count[target]), distance 30."""

    kind = C.LINK

    def __init__(self, source=(), target=()):
        super().__init__()
        self._links = (source, target)
        self._id = None  # link.js:4-6: a node's id is its index
        self.source, self.target = self._unresolved()
        self._strength = None  # default strength
        self._distance = _constant(30.0)
        self._iterations = 1
        self.count = None
        self.bias = None

    def _resolve(self):
        """link.js:41-50: with an id accessor, every endpoint is a node id,
        looked up among id(i) for the nodes (a later node wins a repeated id);
        an unknown id is an error."""
        src, tgt = self._links
        if self._id is None:
            return np.asarray(src, np.int64), np.asarray(tgt, np.int64)
        by_id = {self._id(i): i for i in range(len(self.nodes))}

        def find(v):
            if v not in by_id:
                raise KeyError("node not found: %r" % (v,))
            return by_id[v]

        return (np.array([find(v) for v in src], np.int64),
                np.array([find(v) for v in tgt], np.int64))

    def _unresolved(self):
        """The endpoints as indices before initialize: as given when they are
        indices, empty while they are ids awaiting the node table."""
        try:
            return np.asarray(self._links[0], np.int64), np.asarray(self._links[1], np.int64)
        except (TypeError, ValueError):
            return np.zeros(0, np.int64), np.zeros(0, np.int64)

    def links(self, source=None, target=None):
        """link.js:101-103: the links as resolved node indices, or new ones
        (then the force initializes again)."""
        if source is None and target is None:
            return self.source, self.target
        self._links = (source, target)
        self.source, self.target = self._unresolved()
        if self.nodes is not None:
            self._initialize()
        return self

    def id(self, fn=None):
        """link.js:105-107: fn(i) -> the id of node i; applies at the next
        initialize (as in d3)."""
        if fn is None:
            return self._id
        self._id = fn
        return self

    def _initialize(self):
        self.source, self.target = self._resolve()
        n, m = len(self.nodes), len(self.source)
        src, tgt = self.source, self.target
        count = np.zeros(n, np.int64)
        np.add.at(count, src, 1)
        np.add.at(count, tgt, 1)
        self.count = count
        cs = count[src].astype(np.float64)
        ct = count[tgt].astype(np.float64)
        self.bias = cs / (cs + ct)  # link.js:56-58
        self.slot.bind(self.ctx, n)
        self.slot.count(m)
        if m:
            self.slot.u32(C.SOURCE, m)[:] = src.astype(np.uint32)
            self.slot.u32(C.TARGET, m)[:] = tgt.astype(np.uint32)
            self.slot.f64(C.F2, m)[:] = self.bias
        self._write_strength()
        self._write_distance()

    def _write_strength(self):
        m = len(self.source)
        if self.nodes is None or not m:
            return
        if self._strength is None:  # link.js:30-32
            cs = self.count[self.source].astype(np.float64)
            ct = self.count[self.target].astype(np.float64)
            vals = 1.0 / np.minimum(cs, ct)
        else:
            vals = np.array([float(self._strength(i)) for i in range(m)])
        self.slot.f64(C.F0, m)[:] = vals

    def _write_distance(self):
        m = len(self.source)
        if self.nodes is None or not m:
            return
        self.slot.f64(C.F1, m)[:] = np.array([float(self._distance(i)) for i in range(m)])

    def _push(self):
        self.slot.scalar(C.ITERATIONS, self._iterations)

    def iterations(self, k=_GET):
        """link.js:109-111"""
        if k is _GET:
            return self._iterations
        self._iterations = float(k)
        return self

    def _default_strength(self, i):
        """link.js:30-32: 1 / min(count[source], count[target]) of link i."""
        return 1.0 / min(self.count[self.source[i]], self.count[self.target[i]])

    def strength(self, s=_GET):
        """link.js:113-115 (the default strength function when none was set)."""
        if s is _GET:
            return self._default_strength if self._strength is None else self._strength
        self._strength = _accessor(s)
        self._write_strength()
        return self

    def distance(self, d=_GET):
        """link.js:117-119"""
        if d is _GET:
            return self._distance
        self._distance = _accessor(d)
        self._write_distance()
        return self


class ForceCollide(Force):
    """src/collide.js: radius 1, strength 1, iterations 1; alpha ignored."""

    kind = C.COLLIDE

    def __init__(self, radius=None):
        super().__init__()
        self._radius = _accessor(1.0 if radius is None else radius)
        self._strength = 1.0
        self._iterations = 1.0

    def _initialize(self):
        n = len(self.nodes)
        self.slot.bind(self.ctx, n)
        self.slot.count(n)
        a = self.slot.f64(C.F0, n)
        for i in range(n):
            a[i] = float(self._radius(i))

    def __call__(self, alpha):
        self._push()
        self.slot.run(0.0)

    def _push(self):
        self.slot.scalar(C.STRENGTH, self._strength)
        self.slot.scalar(C.ITERATIONS, self._iterations)

    def radius(self, r=_GET):
        """collide.js:45-47"""
        if r is _GET:
            return self._radius
        self._radius = _accessor(r)
        if self.nodes is not None:
            self._initialize()
        return self

    def strength(self, s=_GET):
        """collide.js:41-43"""
        if s is _GET:
            return self._strength
        self._strength = float(s)
        return self

    def iterations(self, k=_GET):
        """collide.js:37-39"""
        if k is _GET:
            return self._iterations
        self._iterations = float(k)
        return self


class ForceCenter(Force):
    """src/center.js"""

    kind = C.CENTER

    def __init__(self, x=0.0, y=0.0):
        super().__init__()
        self.cx, self.cy, self._strength = float(x), float(y), 1.0

    def __call__(self, alpha):
        self._push()
        self.slot.run(0.0)

    def _push(self):
        self.slot.scalar(C.CX, self.cx)
        self.slot.scalar(C.CY, self.cy)
        self.slot.scalar(C.STRENGTH, self._strength)

    def x(self, v=_GET):
        """center.js:21-23"""
        if v is _GET:
            return self.cx
        self.cx = float(v)
        return self

    def y(self, v=_GET):
        """center.js:25-27"""
        if v is _GET:
            return self.cy
        self.cy = float(v)
        return self

    def strength(self, s=_GET):
        """center.js:29-31"""
        if s is _GET:
            return self._strength
        self._strength = float(s)
        return self


class _ForceAxis(Force):
    """src/x.js, src/y.js: strength 0.1, target 0 (NaN target -> strength 0)."""

    def __init__(self, target=0.0):
        super().__init__()
        self._target = _accessor(target)
        self._strength = _constant(0.1)

    def _initialize(self):
        n = len(self.nodes)
        tz = np.array([float(self._target(i)) for i in range(n)])
        st = np.array([0.0 if math.isnan(tz[i]) else float(self._strength(i)) for i in range(n)])
        self.slot.bind(self.ctx, n)
        self.slot.count(n)
        if n:
            self.slot.f64(C.F0, n)[:] = st
            self.slot.f64(C.F1, n)[:] = tz

    def strength(self, s=_GET):
        """x.js:36-38, y.js:36-38"""
        if s is _GET:
            return self._strength
        self._strength = _accessor(s)
        if self.nodes is not None:
            self._initialize()
        return self

    def _target_of(self, v):
        if v is _GET:
            return self._target
        self._target = _accessor(v)
        if self.nodes is not None:
            self._initialize()
        return self


class ForceX(_ForceAxis):
    kind = C.X

    def x(self, v=_GET):
        """x.js:40-42"""
        return self._target_of(v)


class ForceY(_ForceAxis):
    kind = C.Y

    def y(self, v=_GET):
        """y.js:40-42"""
        return self._target_of(v)


class ForceRadial(Force):
    """src/radial.js"""

    kind = C.RADIAL

    def __init__(self, radius, x=0.0, y=0.0):
        super().__init__()
        self._radius = _accessor(radius)
        self._strength = _constant(0.1)
        self.cx, self.cy = float(x), float(y)

    def _initialize(self):
        n = len(self.nodes)
        rz = np.array([float(self._radius(i)) for i in range(n)])
        st = np.array([0.0 if math.isnan(rz[i]) else float(self._strength(i)) for i in range(n)])
        self.slot.bind(self.ctx, n)
        self.slot.count(n)
        if n:
            self.slot.f64(C.F0, n)[:] = st
            self.slot.f64(C.F1, n)[:] = rz

    def _push(self):
        self.slot.scalar(C.CX, self.cx)
        self.slot.scalar(C.CY, self.cy)

    def strength(self, s=_GET):
        """radial.js:39-41"""
        if s is _GET:
            return self._strength
        self._strength = _accessor(s)
        if self.nodes is not None:
            self._initialize()
        return self

    def radius(self, r=_GET):
        """radial.js:43-45"""
        if r is _GET:
            return self._radius
        self._radius = _accessor(r)
        if self.nodes is not None:
            self._initialize()
        return self

    def x(self, v=_GET):
        """radial.js:47-49"""
        if v is _GET:
            return self.cx
        self.cx = float(v)
        return self

    def y(self, v=_GET):
        """radial.js:51-53"""
        if v is _GET:
            return self.cy
        self.cy = float(v)
        return self


def d3_lcg(seed=1):
    """src/lcg.js: d3's LCG as a Python callable (for host-side draws)."""
    state = [seed & 0xFFFFFFFF]

    def rnd():
        state[0] = (1664525 * state[0] + 1013904223) % 4294967296
        return state[0] / 4294967296

    return rnd


class Simulation:
    """src/simulation.js:17-215 over a core."""

    def __init__(self, nodes, core):
        self.core = core
        self._nodes = nodes
        self._alpha = 1.0
        self._alpha_min = 0.001
        self._alpha_decay = 1 - math.pow(self._alpha_min, 1 / 300)
        self._alpha_target = 0.0
        self._velocity_decay = 0.6
        self._forces = {}  # insertion order = Map order
        self._random = None  # None = d3's lcg() on the device
        # tick() through one sim_tick call (True), or one force_run per force
        # per tick as the reference's facade drives its core (False)
        self.engine_ticks = True
        self._precision = "exact"
        self.ctx = Context(core)
        self.ctx.set_random(None)
        C.check(core.sim_set_lcg(self.ctx.h, 1))
        self._initialize_nodes()

    # simulation.js:91-105
    def _initialize_nodes(self):
        nd = self._nodes
        for i in range(nd.n):
            if not math.isnan(nd.fx[i]):
                nd.x[i] = nd.fx[i]
            if not math.isnan(nd.fy[i]):
                nd.y[i] = nd.fy[i]
            if math.isnan(nd.x[i]) or math.isnan(nd.y[i]):
                radius = INITIAL_RADIUS * math.sqrt(0.5 + i)
                angle = i * INITIAL_ANGLE
                nd.x[i] = radius * math.cos(angle)
                nd.y[i] = radius * math.sin(angle)
            if math.isnan(nd.vx[i]) or math.isnan(nd.vy[i]):
                nd.vx[i] = nd.vy[i] = 0.0
        self.ctx.resize(nd.n)

    def tick(self, iterations=1):
        """simulation.js:49-89. With the device LCG as the random source the
        ticks run in one engine call (sim_tick: the same forces in the same
        order, bit for bit, with the center sums overlapped on a side stream);
        with a randomSource() callback, one force_run per force per tick."""
        if not (0 < iterations):
            return self
        if self._random is None and self.engine_ticks and not self._custom():
            # one engine call: node state up, the ticks, node state down
            ctx = self.ctx
            ctx.bind(self._nodes)
            self._push_forces()
            alpha = C._F64(self._alpha)
            C.check(self.core.sim_tick_sync(ctx.h, int(iterations), alpha, self._alpha_target,
                                            self._alpha_decay, self._velocity_decay, self._order,
                                            self._n_order))
            self._alpha = alpha.value
            ctx.read_back(self._nodes)
            return self
        ctx = self.ctx
        ctx.copy_in(self._nodes)
        ctx.live = True
        try:
            for _ in range(int(iterations)):
                self._alpha += (self._alpha_target - self._alpha) * self._alpha_decay
                for f in self._forces.values():
                    if isinstance(f, Force):
                        f(self._alpha)
                        continue
                    # simulation.js:66-76: a custom force sees the node table
                    # through a copy-out and copy-in around it
                    ctx.live = False
                    ctx.copy_out(self._nodes)
                    try:
                        f(self._alpha)
                    finally:
                        ctx.copy_in(self._nodes)
                        ctx.live = True
                C.check(self.core.sim_integrate(ctx.h, self._velocity_decay))
        finally:
            ctx.live = False
            ctx.copy_out(self._nodes)
        return self

    def _custom(self):
        """Whether a force other than the core's is registered."""
        return any(not isinstance(f, Force) for f in self._forces.values())

    def _draw(self):
        """One draw from the simulation's random source, as the reference hands
        it to a custom force's initialize(nodes, random): the randomSource()
        callable, else d3's LCG, whose state the core keeps (so core jiggles
        and custom forces share one stream, as in simulation.js:22)."""
        if self._random is not None:
            return self._random()
        h = self.ctx.h
        s = (1664525 * int(self.core.sim_get_lcg(h)) + 1013904223) % 4294967296
        C.check(self.core.sim_set_lcg(h, s))
        return s / 4294967296

    def _initialize_force(self, f):
        """simulation.js:107-110: a core force binds its slots; a custom force
        gets initialize(nodes, random) if it has one."""
        if isinstance(f, Force):
            f.initialize(self._nodes, self.ctx)
        elif hasattr(f, "initialize"):
            f.initialize(self._nodes, self._draw)
        return f

    def run(self, ticks):
        """`ticks` ticks in one engine call (sim_tick); bitwise the same as
        `ticks` calls of tick(1). Needs the device LCG random source; with a
        randomSource() callback it falls back to tick(ticks)."""
        if self._random is not None or self._custom():
            return self.tick(ticks)
        self.device_begin()
        self.device_ticks(ticks)
        self.device_end()
        return self

    def device_begin(self):
        """Node state to the device and every force's scalars pushed, so that
        device_ticks() can run ticks with no host transfer. Core forces only: a
        custom force runs through tick()."""
        if self._custom():
            raise ValueError("a custom force runs through tick(), not the engine's sim_tick")
        ctx = self.ctx
        ctx.copy_in(self._nodes)
        self._push_forces()

    def _push_forces(self):
        """Every force's scalars (sent only when changed) and the force order
        for sim_tick (rebuilt only when the forces changed). Skipped when no
        force attribute, force handle or precision setting moved since the
        last push."""
        ctx = self.ctx
        handles = tuple(f.slot.fh for f in self._forces.values())
        prec = tuple(ctx.precision.items()) if ctx.precision else None
        key = (_FORCE_GEN[0], handles, prec)
        if getattr(self, "_push_key", None) == key:
            return
        for f in self._forces.values():
            f._push()
            s = f.slot
            s.scalar(C.PRECISION, ctx.precision["form"] if ctx.precision else 0)
            if ctx.precision:
                s.scalar(C.ORDER, ctx.precision["order"])
                s.scalar(C.OPENING, ctx.precision["opening"])
        if getattr(self, "_order_key", None) != handles:
            self._order = (C._U32 * max(1, len(handles)))(*handles)
            self._n_order = len(handles)
            self._order_key = handles
        self._push_key = (_FORCE_GEN[0], handles, prec)

    def device_ticks(self, ticks):
        """`ticks` ticks on the device (sim_tick); returns their device ms.
        collide and center get alpha 0 from the facade and ignore it in the
        core, so one alpha per tick for every force is equivalent."""
        alpha = C._F64(self._alpha)
        C.check(self.core.sim_tick(self.ctx.h, int(ticks), alpha, self._alpha_target,
                                   self._alpha_decay, self._velocity_decay, self._order,
                                   self._n_order))
        self._alpha = alpha.value
        return self.core.sim_last_tick_ms(self.ctx.h)

    def device_end(self):
        self.ctx.copy_out(self._nodes)

    def nodes(self, nodes=None):
        if nodes is None:
            return self._nodes
        self._nodes = nodes
        self._initialize_nodes()
        for f in self._forces.values():
            self._initialize_force(f)
        return self

    def alpha(self, a=None):
        if a is None:
            return self._alpha
        self._alpha = float(a)
        return self

    def alphaMin(self, a=None):
        if a is None:
            return self._alpha_min
        self._alpha_min = float(a)
        return self

    def alphaDecay(self, a=None):
        if a is None:
            return self._alpha_decay
        self._alpha_decay = float(a)
        return self

    def alphaTarget(self, a=None):
        if a is None:
            return self._alpha_target
        self._alpha_target = float(a)
        return self

    def velocityDecay(self, a=None):
        if a is None:
            return 1 - self._velocity_decay
        self._velocity_decay = 1 - float(a)
        return self

    def randomSource(self, fn=None):
        """simulation.js:149-151: a callable drawn for every jiggle, in d3's order."""
        if fn is None:
            return self._random
        self._random = fn
        self.ctx.set_random(fn)
        for f in self._forces.values():
            self._initialize_force(f)
        return self

    def force(self, name, f="__get__"):
        if f == "__get__":
            return self._forces.get(name)
        if f is None:
            self._forces.pop(name, None)
        else:
            self._forces[name] = self._initialize_force(f)
        return self

    # fast-mode forms of the many-body force: the PRECISION scalar the core gets
    FORMS = {"plain": 1, "bf16x3": 2, "learned": 3}

    def precision(self, mode=None, order=None, opening=None, form="plain"):
        """simulation.js:187-200. `form` (no counterpart in the reference)
        picks the fast many-body force: "plain" is the reference's FP64 FMM
        bit for bit; "bf16x3" the tensor-core FMM (M2L as BF16x3 contractions
        on geometric cells, FP32 near field; order up to 15, opening 1 to 2);
        "learned" order 4 with the learned per-leaf correction."""
        if mode is None:
            return self._precision
        if mode not in ("exact", "fast"):
            raise ValueError('precision must be "exact" or "fast"')
        if form not in self.FORMS:
            raise ValueError("form must be one of " + ", ".join(sorted(self.FORMS)))
        self._precision = mode
        if mode == "fast":
            o = order if order else 8
            self.ctx.precision = {"order": min(24, max(1, round(float(o)))),
                                  "opening": max(1.01, float(opening) if opening else 1.5),
                                  "form": self.FORMS[form]}
        else:
            self.ctx.precision = None
        return self

    def learned(self, params, tolerance=1e-5, samples=64, hold=16):
        """Installs the learned form's network (5,122 floats, learned.py) with
        its sampled check: each checked tick the order-4 + network kick is
        compared with an FP64 direct sum on `samples` nodes, and when the RMS
        exceeds `tolerance` the tick runs the plain form instead, and so do
        the next `hold` ticks before the network is checked again. No
        counterpart in the reference."""
        import numpy as np
        p = np.ascontiguousarray(params, np.float32)
        C.check(self.ctx.core.sim_set_learned(self.ctx.h, p.ctypes.data, len(p), float(tolerance),
                                              int(samples), int(hold)))
        return self

    def threads(self, k="__get__"):
        """simulation.js:205-215: the reference's cap on CPU workers per tick.
        Ticks run on the GPU here: the setter is kept for compatibility and
        the getter reports 0 workers used (as the reference's inlined core)."""
        if k == "__get__":
            return 0
        if k is None:
            self._threads = None
            return self
        v = float(k)  # Math.max(0, Math.floor(+k) || 0)
        if v != v:
            v = 0.0
        elif not math.isinf(v):
            v = float(math.floor(v))
        self._threads = max(0.0, v)
        return self

    def find(self, x, y, radius=None):
        """simulation.js:157-178 through the core (sim_find, a reduction on
        the device): the index of the closest node with d2 < radius^2 (the
        lowest index among equal d2), or None."""
        ctx = self.ctx
        ctx.copy_in(self._nodes)
        out = C._U32(0)
        r = math.inf if radius is None else float(radius)
        C.check(self.core.sim_find(ctx.h, float(x), float(y), r, ctypes.byref(out)))
        return None if out.value == 0xFFFFFFFF else int(out.value)

    def close(self):
        self.ctx.close()


def forceSimulation(nodes=None, core=None):
    if core is None:
        from . import cuda_core

        core = cuda_core()
    if nodes is None:
        nodes = Nodes(0)
    return Simulation(nodes, core)


def forceManyBody():
    return ForceManyBody()


def forceLink(source=(), target=()):
    return ForceLink(source, target)


def forceCollide(radius=None):
    return ForceCollide(radius)


def forceCenter(x=0.0, y=0.0):
    return ForceCenter(x, y)


def forceX(x=0.0):
    return ForceX(x)


def forceY(y=0.0):
    return ForceY(y)


def forceRadial(radius, x=0.0, y=0.0):
    return ForceRadial(radius, x, y)
