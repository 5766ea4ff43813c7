"""Accuracy of the fast many-body forms: the kick of one tick against an FP64
direct sum of d3's pair formula, as the reference measures its FMM
(test/fast/error-test.js:44-70, src/core/bench.zig:80-104, fmm.zig:913-1000):

    RMS = sqrt( sum_i |v_i - v_ref_i|^2 / sum_i |v_ref_i|^2 )

over seeded target nodes. The direct sum runs on the GPU in FP64 (torch),
target rows against all sources, with distanceMin's clamp l = sqrt(dmin2 l)
below dmin2; coincident source/target pairs (where d3 draws a jiggle) add
nothing, so targets that have an exact duplicate are left out of the sample.
"""

import numpy as np


def many_body_kick(pkg, core, xs, ys, strength=-30.0, form="plain", order=8, opening=1.5,
                   distance_min=1.0):
    """Runs one tick of a simulation holding only forceManyBody, from zero
    velocity; returns (kick, alpha): the velocity the force added (before the
    velocity decay of the integration) and the alpha it ran with."""
    n = len(xs)
    nodes = pkg.Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody().strength(strength).distanceMin(distance_min))
    sim.precision("fast", order=order, opening=opening, form=form)
    sim.tick()
    alpha = sim.alpha()
    decay = 1 - sim.velocityDecay()
    kick = np.stack([np.asarray(nodes.vx) / decay, np.asarray(nodes.vy) / decay], 1)
    sim.close()
    return kick, alpha


def sample_targets(xs, ys, count, seed=7):
    """`count` seeded target indices, none of which shares its exact position
    with another node."""
    n = len(xs)
    rng = np.random.default_rng(seed)
    order = rng.permutation(n)
    key = np.asarray(xs, np.float64) + 1j * np.asarray(ys, np.float64)
    _, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    unique = cnt[inv] == 1
    return order[unique[order]][:count].astype(np.int64)


def direct_kick(xs, ys, s_alpha, targets, distance_min2=1.0, chunk=64):
    """FP64 direct sum of d3's pair formula on the GPU: for each target i,
    sum_j s_j alpha (x_j - x_i, y_j - y_i) / l_ij with l = d^2, clamped to
    sqrt(dmin2 l) below dmin2, j != i and coincident pairs skipped.
    s_alpha: strength x alpha per node."""
    import torch

    dev = torch.device("cuda")
    X = torch.from_numpy(np.ascontiguousarray(xs, np.float64)).to(dev)
    Y = torch.from_numpy(np.ascontiguousarray(ys, np.float64)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(s_alpha, np.float64)).to(dev)
    out = torch.zeros(len(targets), 2, dtype=torch.float64, device=dev)
    for k0 in range(0, len(targets), chunk):
        idx = torch.from_numpy(np.asarray(targets[k0:k0 + chunk], np.int64)).to(dev)
        dx = X[None, :] - X[idx, None]
        dy = Y[None, :] - Y[idx, None]
        l = dx * dx + dy * dy
        l = torch.where(l < distance_min2, torch.sqrt(distance_min2 * l), l)
        w = torch.where(l > 0, S[None, :] / torch.where(l > 0, l, torch.ones_like(l)),
                        torch.zeros_like(l))
        out[k0:k0 + chunk, 0] = (dx * w).sum(1)
        out[k0:k0 + chunk, 1] = (dy * w).sum(1)
    return out.cpu().numpy()


def rms(kick, ref, targets):
    """sqrt(sum |kick - ref|^2 / sum |ref|^2) over the targets."""
    err = kick[targets] - ref
    return float(np.sqrt((err * err).sum() / (ref * ref).sum()))
