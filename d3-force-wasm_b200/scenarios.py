"""Seeded workloads: the reference's test scenarios and the benchmark configs.

`generator` is the reference's data generator (test/parity/scenarios.js:7-16,
a mulberry32-style hash of a counter); the `fast_*` layouts restate
test/threads/scenarios.js:13-56 (inputs built from correctly rounded
arithmetic only). `exact_graph` builds the exact-mode benchmark workloads
(n nodes without positions so d3's phyllotaxis start applies, m = 2n links
drawn from d3's LCG, optional coincident / near-duplicate / pinned nodes).
"""

import hashlib
import math

import numpy as np

from .simulation import Nodes, d3_lcg

M32 = 0xFFFFFFFF


def _imul(a, b):
    return (a * b) & M32


def generator(seed):
    """test/parity/scenarios.js:7-16"""
    s = [seed & M32]

    def r():
        s[0] = (s[0] + 0x6D2B79F5) & M32
        t = s[0]
        t = _imul(t ^ (t >> 15), t | 1)
        t = t ^ ((t + _imul(t ^ (t >> 7), t | 61)) & M32)
        return ((t ^ (t >> 14)) & M32) / 4294967296

    return r


def _disk(r, cx, cy, radius):
    """test/threads/scenarios.js:13-17"""
    while True:
        x = 2 * r() - 1
        y = 2 * r() - 1
        if not (x * x + y * y > 1):
            return cx + radius * x, cy + radius * y


def _spiral(n):
    """test/threads/scenarios.js:21-29"""
    c, s = -0.7373688780783197, 0.6754902942615238
    xs, ys = [], []
    u, v = 1.0, 0.0
    for i in range(n):
        radius = 10 * math.sqrt(0.5 + i)
        xs.append(radius * u)
        ys.append(radius * v)
        u, v = u * c - v * s, u * s + v * c
    return xs, ys


def _layout(name, r):
    """test/threads/scenarios.js:31-37"""
    xs, ys = [], []
    if name == "uniform 4000":
        for _ in range(4000):
            x = 1000 * (r() - 0.5)
            y = 1000 * (r() - 0.5)
            xs.append(x)
            ys.append(y)
    elif name == "three clusters 6000":
        for i in range(6000):
            x, y = _disk(r, (0, 400, -300)[i % 3], (0, 100, 350)[i % 3], 120)
            xs.append(x)
            ys.append(y)
    elif name == "spiral 8000":
        xs, ys = _spiral(8000)
    elif name == "grid 2500 with exact zero deltas":
        for i in range(2500):
            xs.append(12.0 * (i % 50))
            ys.append(12.0 * (i // 50))
    elif name == "dense sub-unit cluster 3000":
        for _ in range(3000):
            x = 20 * r()
            y = 20 * r()
            xs.append(x)
            ys.append(y)
    else:
        raise KeyError(name)
    return xs, ys


FAST_SCENARIOS = ("uniform 4000", "three clusters 6000", "spiral 8000",
                  "grid 2500 with exact zero deltas", "dense sub-unit cluster 3000")
CHECKPOINTS = (1, 10, 100, 300)


def fast_scenario(name, seed=1):
    """Nodes and links of a large scenario (test/threads/scenarios.js:39-56):
    charge, link (i -> floor(r() n)), collide(3), center; precision 'fast'."""
    r = generator(seed)
    xs, ys = _layout(name, r)
    n = len(xs)
    src = np.arange(n, dtype=np.int64)
    tgt = np.array([math.floor(r() * n) for _ in range(n)], np.int64)
    return Nodes(n, x=xs, y=ys), src, tgt


def setup_fast_scenario(pkg, core, name, mode="fast", seed=1):
    nodes, src, tgt = fast_scenario(name, seed)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.force("link", pkg.forceLink(src, tgt))
    sim.force("collide", pkg.forceCollide(3))
    sim.force("center", pkg.forceCenter())
    if mode:
        sim.precision(mode)
    return nodes, sim


def digest(nodes):
    """test/threads/digest.js:6-13: SHA-256 of interleaved x, y, vx, vy f64."""
    a = np.empty(4 * nodes.n, np.float64)
    a[0::4], a[1::4], a[2::4], a[3::4] = nodes.x, nodes.y, nodes.vx, nodes.vy
    return hashlib.sha256(a.astype("<f8").tobytes()).hexdigest()


def lcg_links(n, m, seed=1):
    """m links with endpoints floor(u n) from d3's LCG, redrawn on a self-loop."""
    rnd = d3_lcg(seed)
    src = np.empty(m, np.int64)
    tgt = np.empty(m, np.int64)
    for k in range(m):
        s = math.floor(rnd() * n)
        t = math.floor(rnd() * n)
        while t == s:
            t = math.floor(rnd() * n)
        src[k], tgt[k] = s, t
    return src, tgt


def exact_graph(n, m, coincident=0.0, near=0.0, pinned=0.0, seed=1):
    """The exact-mode benchmark workload. Nodes start without positions, so
    d3's phyllotaxis places them (simulation.js:96-100); then a fraction of
    nodes is moved onto exact copies of other nodes' positions, a fraction to
    offsets below 1e-12 from other nodes, and a fraction pinned (fx, fy) at
    its start. Links: `lcg_links`. Returns (nodes, src, tgt) with positions
    filled in (the phyllotaxis step is applied here so every node is set)."""
    nodes = Nodes(n)
    for i in range(n):
        radius = 10 * math.sqrt(0.5 + i)
        angle = i * (math.pi * (3 - math.sqrt(5)))
        nodes.x[i] = radius * math.cos(angle)
        nodes.y[i] = radius * math.sin(angle)
    nodes.vx[:] = 0
    nodes.vy[:] = 0
    rnd = d3_lcg(seed * 7919 + 17)
    k_co, k_near, k_pin = int(coincident * n), int(near * n), int(pinned * n)
    chosen = set()

    def pick():
        while True:
            i = math.floor(rnd() * n)
            if i not in chosen:
                chosen.add(i)
                return i

    for _ in range(k_co):
        i, j = pick(), math.floor(rnd() * n)
        nodes.x[i], nodes.y[i] = nodes.x[j], nodes.y[j]
    for _ in range(k_near):
        i, j = pick(), math.floor(rnd() * n)
        nodes.x[i] = nodes.x[j] + (rnd() - 0.5) * 1e-12
        nodes.y[i] = nodes.y[j] + (rnd() - 0.5) * 1e-12
    for _ in range(k_pin):
        i = pick()
        nodes.fx[i], nodes.fy[i] = nodes.x[i], nodes.y[i]
    src, tgt = lcg_links(n, m, seed)
    return nodes, src, tgt


def setup_exact(pkg, core, n, m, collide_radius=None, coincident=0.0, near=0.0, pinned=0.0,
                seed=1):
    """forceManyBody(-30, theta 0.9), forceLink(distance 30, default strength),
    forceCenter(0, 0) and optionally forceCollide(radius) on `exact_graph`."""
    nodes, src, tgt = exact_graph(n, m, coincident, near, pinned, seed)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody().theta(0.9))
    sim.force("link", pkg.forceLink(src, tgt))
    if collide_radius is not None:
        sim.force("collide", pkg.forceCollide(collide_radius))
    sim.force("center", pkg.forceCenter(0, 0))
    return nodes, sim
