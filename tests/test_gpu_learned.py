"""The learned form of the fast many-body force on the B200 (no reference
counterpart): a network trained on the GPU by the package's own kernels on
order-4 vs order-12 pairs of mixture layouts, then applied to a held-out
layout. Judged as the FMM is judged: RMS of the kick against an FP64 direct
sum on seeded targets (test/fast/error-test.js:44-70)."""

import importlib

import numpy as np
import pytest

import helpers as H

pkg = H.pkg
acc = importlib.import_module("d3-force-wasm_b200.accuracy")
learned = importlib.import_module("d3-force-wasm_b200.learned")
pytestmark = pytest.mark.gpu

N = 100000


@pytest.fixture(scope="module")
def trained(gcore):
    layouts = [learned.mixture_layout(N, seed)[:2] for seed in range(100, 140)]
    X, Y = learned.training_pairs(gcore, layouts)
    params, losses = learned.train(gcore, X, Y, steps=1500, batch=4096)
    return params, losses, len(X)


def _kick(gcore, xs, ys, form, order, params=None, tol=1e9):
    n = len(xs)
    nodes = pkg.Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=gcore)
    sim.force("charge", pkg.forceManyBody())
    sim.precision("fast", order=order, opening=1.5, form=form)
    if params is not None:
        sim.learned(params, tolerance=tol, samples=64)
    sim.tick()
    alpha = sim.alpha()
    kick = np.stack([np.asarray(nodes.vx), np.asarray(nodes.vy)], 1) / 0.6
    stats = [gcore.sim_stat(sim.ctx.h, 50 + k) for k in range(3)]
    sim.close()
    return kick, alpha, stats


def test_gpu_learned_training_lowers_the_loss(trained):
    params, losses, n = trained
    assert n > 100000
    assert np.all(np.isfinite(params))
    assert losses[-50:].mean() < losses[:10].mean()


def test_gpu_learned_correction_measured_against_plain_order_4(gcore, trained):
    """What the trained network gains over the order-4 form without it, on a
    held-out layout (the check is disabled so the corrected kick is applied):
    both RMS errors against the FP64 direct sum are printed. The correction
    of a leaf's L'_0 is bounded at about a third of the order-4 error (the
    rest varies inside the leaf), and the residual is nearly unpredictable
    from the leaf's expansion, so the measured gain is small; the test checks
    that the network does no material harm (the sampled check and the
    fallback keep the tolerance in any case)."""
    params = trained[0]
    xs, ys, _ = learned.mixture_layout(N, 999)
    tg = acc.sample_targets(xs, ys, 2048)
    k4, alpha, _ = _kick(gcore, xs, ys, "bf16x3", 4)
    kl, alpha2, st = _kick(gcore, xs, ys, "learned", 8, params)
    assert alpha == alpha2 and st[1] == 0  # applied, no fallback
    ref = acc.direct_kick(xs, ys, np.full(N, -30.0 * alpha), tg)
    r4, rl = acc.rms(k4, ref, tg), acc.rms(kl, ref, tg)
    print("order 4 RMS %.4g, learned %.4g, gain %.2f%%" % (r4, rl, 100 * (1 - rl / r4)))
    assert rl <= 1.05 * r4


def test_gpu_learned_falls_back_to_plain_form(gcore, trained):
    """A check that cannot pass (tolerance 1e-12) hands the tick to the
    plain form at order 8: bit for bit its result, one fallback counted."""
    params = trained[0]
    xs, ys, _ = learned.mixture_layout(30000, 5)
    k8, _, _ = _kick(gcore, xs, ys, "bf16x3", 8)
    kf, _, st = _kick(gcore, xs, ys, "learned", 8, params, tol=1e-12)
    assert st[0] == 1 and st[1] == 1 and st[2] > 1e-12
    assert np.array_equal(kf.view(np.uint64), k8.view(np.uint64))
