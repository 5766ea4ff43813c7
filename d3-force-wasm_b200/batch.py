"""Batched fast mode (no reference counterpart): thousands of independent
graphs ticked together, one persistent kernel launch per tick, a run of
ticks captured in a CUDA graph, launch shape autotuned (csrc/batch.cu).

    graphs = batch_workload(2048, seed=1)
    b = Batch(core, graphs)
    b.autotune()
    ms = b.run(300)              # 300 ticks, one CUDA graph
    b.close()

The workload of the batched configuration: node counts log-uniform in
[64, 16384]; half the graphs with m = 2n uniform random links, half a
stochastic block model with 8 communities and mean degree 4 (p_in / p_out
20); d3's phyllotaxis start positions (simulation.js:96-100).

Across GPUs the graphs shard with no collective: `shard(sizes, world)`
gives each rank a greedy size-balanced share.
"""

import ctypes
import math

import numpy as np

from . import core as C

_U32P = ctypes.POINTER(ctypes.c_uint32)
_F32P = ctypes.POINTER(ctypes.c_float)
_F64P = ctypes.POINTER(ctypes.c_double)


def _bind(lib):
    sig = {
        "batch_create": (ctypes.c_uint32, [ctypes.c_uint32, _U32P, _U32P, _U32P, _U32P, _F32P,
                                           _F32P]),
        "batch_destroy": (ctypes.c_int32, [ctypes.c_uint32]),
        "batch_set_shape": (ctypes.c_int32, [ctypes.c_uint32] * 4),
        "batch_run": (ctypes.c_int32, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _F64P]),
        "batch_kick": (ctypes.c_int32, [ctypes.c_uint32, _F32P, _F64P]),
        "batch_read": (ctypes.c_int32, [ctypes.c_uint32, _F32P, _F32P, _F32P, _F32P]),
        "batch_autotune": (ctypes.c_int32, [ctypes.c_uint32, ctypes.c_uint32, _F64P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def phyllotaxis(n):
    """d3's start positions (simulation.js:96-100), as float64."""
    i = np.arange(n, dtype=np.float64)
    r = 10 * np.sqrt(0.5 + i)
    a = i * math.pi * (3 - math.sqrt(5))
    return r * np.cos(a), r * np.sin(a)


def batch_workload(graphs=2048, seed=1, nmin=64, nmax=16384):
    """[(n, src, tgt)] for the batched configuration (seeded)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), graphs)).astype(np.int64)
    out = []
    for g, n in enumerate(sizes):
        n = int(max(nmin, min(nmax, n)))
        if g % 2 == 0:  # uniform random links, m = 2n
            src = rng.integers(0, n, 2 * n)
            tgt = (src + 1 + rng.integers(0, n - 1, 2 * n)) % n
        else:  # SBM: 8 communities, mean degree 4, p_in / p_out = 20
            lab = rng.integers(0, 8, n)
            m = 2 * n
            counts = np.bincount(lab, minlength=8).astype(np.float64)
            s_in = (counts * (counts - 1) / 2).sum()
            s_out = n * (n - 1) / 2 - s_in
            p_int = 20 * s_in / (20 * s_in + s_out)
            order = np.argsort(lab, kind="stable")
            starts = np.concatenate([[0], np.cumsum(counts).astype(np.int64)])
            src = rng.integers(0, n, m)
            internal = rng.random(m) < p_int
            li = lab[src[internal]]
            tgt = np.empty(m, np.int64)
            tgt[internal] = order[starts[li] + (rng.random(internal.sum()) *
                                                counts[li]).astype(np.int64)]
            tgt[~internal] = rng.integers(0, n, (~internal).sum())
            same = src == tgt
            tgt[same] = (tgt[same] + 1) % n
        out.append((n, src.astype(np.uint32), tgt.astype(np.uint32)))
    return out


def shard(sizes, world):
    """Greedy size balance: graphs largest first, each to the rank with the
    least work so far (ties to the lower rank). Returns a list of graph index
    lists, one per rank."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for g in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(g)
        load[r] += sizes[g]
    return parts


class Batch:
    """The device batch of `graphs` = [(n, src, tgt)] on the CUDA engine."""

    def __init__(self, core, graphs, positions=None):
        """positions: optional [(x, y)] per graph; d3's phyllotaxis start
        otherwise."""
        self.lib = _bind(core.lib)
        counts = np.array([g[0] for g in graphs], np.uint32)
        links = np.array([len(g[1]) for g in graphs], np.uint32)
        src = np.concatenate([g[1] for g in graphs]).astype(np.uint32)
        tgt = np.concatenate([g[2] for g in graphs]).astype(np.uint32)
        xs, ys = [], []
        for g, (n, _, _) in enumerate(graphs):
            x, y = positions[g] if positions is not None else phyllotaxis(n)
            xs.append(np.asarray(x, np.float64))
            ys.append(np.asarray(y, np.float64))
        self.x0 = np.concatenate(xs).astype(np.float32)
        self.y0 = np.concatenate(ys).astype(np.float32)
        self.counts = counts
        self.offsets = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        self.nodes = int(self.offsets[-1])
        u = lambda a: a.ctypes.data_as(_U32P)  # noqa: E731
        f = lambda a: a.ctypes.data_as(_F32P)  # noqa: E731
        self.h = self.lib.batch_create(len(graphs), u(counts), u(links), u(src), u(tgt),
                                       f(self.x0), f(self.y0))
        if not self.h:
            raise C.CoreError(C.OUT_OF_MEMORY)

    def set_shape(self, threads, per_sm, leaf):
        C.check(self.lib.batch_set_shape(self.h, threads, per_sm, leaf))

    def autotune(self, ticks=3):
        out = (ctypes.c_double * 4)()
        C.check(self.lib.batch_autotune(self.h, ticks, out))
        return {"threads": int(out[0]), "ctas_per_sm": int(out[1]), "leaf_size": int(out[2]),
                "ms_per_tick": out[3]}

    def run(self, ticks, graph=True):
        ms = ctypes.c_double(0)
        C.check(self.lib.batch_run(self.h, ticks, 1 if graph else 0, ctypes.byref(ms)))
        return ms.value

    def kick(self):
        out = np.zeros(2 * self.nodes, np.float32)
        al = ctypes.c_double(0)
        C.check(self.lib.batch_kick(self.h, out.ctypes.data_as(_F32P), ctypes.byref(al)))
        return out.reshape(-1, 2), al.value

    def read(self):
        arrs = [np.zeros(self.nodes, np.float32) for _ in range(4)]
        C.check(self.lib.batch_read(self.h, *[a.ctypes.data_as(_F32P) for a in arrs]))
        return arrs

    def close(self):
        if self.h:
            self.lib.batch_destroy(self.h)
            self.h = 0


def graph_rms(batch, kick, alpha, graphs, targets=256, seed=3):
    """Per-graph RMS of the many-body kick against an FP64 direct sum on
    `targets` seeded nodes of each listed graph (all its nodes when fewer),
    at the batch's current positions. Returns an array over `graphs`."""
    import torch

    x, y, _, _ = batch.read()
    rng = np.random.default_rng(seed)
    out = []
    for g in graphs:
        o, n = int(batch.offsets[g]), int(batch.counts[g])
        xs = torch.from_numpy(x[o:o + n].astype(np.float64)).cuda()
        ys = torch.from_numpy(y[o:o + n].astype(np.float64)).cuda()
        tg = rng.choice(n, min(n, targets), replace=False)
        ti = torch.from_numpy(tg).cuda()
        dx = xs[None, :] - xs[ti, None]
        dy = ys[None, :] - ys[ti, None]
        l = dx * dx + dy * dy
        l = torch.where(l < 1.0, torch.sqrt(l), l)
        w = torch.where(l > 0, -30.0 * alpha / torch.where(l > 0, l, torch.ones_like(l)),
                        torch.zeros_like(l))
        ref = torch.stack([(dx * w).sum(1), (dy * w).sum(1)], 1).cpu().numpy()
        err = kick[o + tg] - ref
        out.append(float(np.sqrt((err * err).sum() / (ref * ref).sum())))
    return np.array(out)
