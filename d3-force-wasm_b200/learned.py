"""The learned form of the fast many-body force (no reference counterpart):
an order-4 tensor-core FMM whose leaf-centre local coefficient L'_0 is
corrected by a small network, trained on the GPU by this package's own
kernels (csrc/mlp.cu) on pairs of order-4 and order-12 runs.

Per leaf the network sees 12 numbers (csrc/fmm_tc.cu, k_tc_features): the
order-4 local expansion L'_1 .. L'_4 over its scale sc = |(L'_0 .. L'_4)|,
the level / 16, the point count / 32 and the points' mean offset from the
cell centre; it predicts (L'_0 at order 12 - L'_0 at order 4) / sc x 1000.

    layouts = [mixture_layout(n, seed) for seed in range(200)]
    X, Y = training_pairs(core, layouts)
    params = train(core, X, Y)
    sim.learned(params)          # then precision("fast", form="learned")

The configuration it serves: n nodes in a mixture of 64 Gaussian clusters
(sigma uniform in [50, 500], weights Dirichlet(1), centres uniform in the
1e4 square) with m = 2n links of a stochastic block model (communities = the
clusters, p_in / p_out = 20, mean degree 4).
"""

import ctypes

import numpy as np

from . import core as C
from .simulation import Nodes, forceManyBody, forceSimulation

TARGET_SCALE = 1000.0  # the network's output unit (LEARN_TARGET_SCALE in fmm_tc.cu)
N_IN, N_HID, N_OUT = 12, 64, 2
N_PARAMS = N_HID * N_IN + N_HID + N_HID * N_HID + N_HID + N_OUT * N_HID + N_OUT


def mixture_layout(n, seed, clusters=64, extent=1e4, sigma=(50.0, 500.0)):
    """n positions from a seeded mixture of `clusters` Gaussians."""
    rng = np.random.default_rng(seed)
    cx = rng.random(clusters) * extent
    cy = rng.random(clusters) * extent
    sg = sigma[0] + (sigma[1] - sigma[0]) * rng.random(clusters)
    w = rng.dirichlet(np.ones(clusters))
    lab = rng.choice(clusters, size=n, p=w)
    xs = cx[lab] + sg[lab] * rng.standard_normal(n)
    ys = cy[lab] + sg[lab] * rng.standard_normal(n)
    return xs, ys, lab


def sbm_links(labels, seed, mean_degree=4, ratio=20.0):
    """m = n * mean_degree / 2 links of a stochastic block model over the
    communities `labels`, with p_in / p_out = ratio: a link is internal with
    probability ratio * S_in / (ratio * S_in + S_out) (S_in, S_out the counts
    of internal and external node pairs); endpoints uniform among the allowed
    pairs; no self-loops."""
    rng = np.random.default_rng(seed + 7919)
    n = len(labels)
    m = n * mean_degree // 2
    counts = np.bincount(labels)
    s_in = float((counts.astype(np.float64) * (counts - 1)).sum() / 2)
    s_all = n * (n - 1) / 2
    s_out = s_all - s_in
    p_int = ratio * s_in / (ratio * s_in + s_out)
    order = np.argsort(labels, kind="stable")
    starts = np.concatenate([[0], np.cumsum(counts)])
    internal = rng.random(m) < p_int
    src = rng.integers(0, n, m)
    tgt = np.empty(m, np.int64)
    # internal: the target from the source's community
    li = labels[src[internal]]
    size = counts[li]
    off = (rng.random(internal.sum()) * size).astype(np.int64)
    tgt[internal] = order[starts[li] + off]
    # external: any node (a same-community pick is kept; it is rare)
    tgt[~internal] = rng.integers(0, n, (~internal).sum())
    same = src == tgt
    tgt[same] = (tgt[same] + 1) % n
    return src, tgt


def leaf_rows(core, xs, ys, order, alpha=1.0):
    """One fast many-body pass of the tensor-core form at `order` over the
    positions (zero velocities): the per-leaf rows of sim_fmm_leaves, as an
    (leaves, 16) float array in cell order."""
    n = len(xs)
    nodes = Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = forceSimulation(nodes, core=core)
    mb = forceManyBody()
    sim.force("charge", mb)
    sim.precision("fast", order=order, opening=1.5, form="bf16x3")
    ctx = sim.ctx
    ctx.copy_in(nodes)
    mb._push()  # theta, distanceMin / distanceMax: the force's scalars
    mb.slot.run(alpha)
    cells = core.sim_fmm_leaves(ctx.h, None, 0)
    rows = np.zeros((max(cells, 1), 16), np.float32)
    got = core.sim_fmm_leaves(ctx.h, rows.ctypes.data, cells)
    sim.close()
    if got < 0:
        raise C.CoreError(got)
    rows = rows[:cells]
    leaf = rows[:, 15].view(np.int32) >= 0
    return rows[leaf]


def training_pairs(core, layouts):
    """(X, Y) float32 arrays from order-4 and order-12 passes over each
    layout (xs, ys): X the order-4 leaf inputs, Y the scaled difference of
    L'_0."""
    xs_all, ys_all = [], []
    for xs, ys in layouts:
        lo = leaf_rows(core, xs, ys, 4)
        hi = leaf_rows(core, xs, ys, 12)
        if len(lo) != len(hi):
            raise RuntimeError("order 4 and order 12 built different trees")
        sc = lo[:, 14:15].astype(np.float64)
        y = (hi[:, 12:14].astype(np.float64) - lo[:, 12:14]) / sc * TARGET_SCALE
        ok = np.isfinite(y).all(1) & (sc[:, 0] > 0)
        xs_all.append(lo[ok, :12])
        ys_all.append(y[ok].astype(np.float32))
    return np.concatenate(xs_all), np.concatenate(ys_all)


def init_params(seed=0):
    """He-scaled random weights, zero biases (the float vector's layout)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    o = 0
    for fan_in, fan_out in ((N_IN, N_HID), (N_HID, N_HID), (N_HID, N_OUT)):
        p[o:o + fan_in * fan_out] = rng.standard_normal(fan_in * fan_out) * np.sqrt(2.0 / fan_in)
        o += fan_in * fan_out + fan_out
    return p


def _bind(lib):
    f = ctypes.POINTER(ctypes.c_float)
    lib.d3_mlp_train.restype = ctypes.c_int32
    lib.d3_mlp_train.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, f, f]
    return lib


def train(core, X, Y, steps=3000, batch=8192, lr=2e-3, seed=0):
    """Trains the network on the GPU (d3_mlp_train: this package's forward,
    backward and Adam kernels) from He-initialised weights; the samples are
    shuffled once and walked in batches. Returns (params, per-step losses)."""
    import torch

    lib = _bind(core.lib)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(X))
    tx = torch.from_numpy(np.ascontiguousarray(X[perm], np.float32)).cuda()
    ty = torch.from_numpy(np.ascontiguousarray(Y[perm], np.float32)).cuda()
    params = init_params(seed)
    losses = np.zeros(steps, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    rc = lib.d3_mlp_train(tx.data_ptr(), ty.data_ptr(), len(X), batch, steps, lr,
                          params.ctypes.data_as(fp), losses.ctypes.data_as(fp))
    if rc != 0:
        raise C.CoreError(rc)
    return params, losses
