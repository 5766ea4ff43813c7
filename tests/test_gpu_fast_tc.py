"""The tensor-core FMM (precision form "bf16x3") on the B200, judged as the
reference judges its fast many-body force: RMS of one tick's kick against an
FP64 direct sum of d3's pair formula (test/fast/error-test.js:44-70,
fmm.zig:913-1000), on seeded targets. The reference's own FMM at order 8,
opening 1.5 reaches about 2e-6 on such layouts; the bound here is the
precision forms' tolerance, RMS <= 1e-5, at that order and opening."""

import importlib

import numpy as np
import pytest

import helpers as H

pkg = H.pkg
acc = importlib.import_module("d3-force-wasm_b200.accuracy")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def _uniform(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random(n) * 1e4, rng.random(n) * 1e4


def _clusters(n, seed):
    """A mixture of 16 Gaussian clusters of widths 20-400 in a 1e4 square: an
    adaptive tree whose leaves sit at many levels (coarse-leaf and
    finer-cell lists in use)."""
    rng = np.random.default_rng(seed)
    k = 16
    cx, cy = rng.random(k) * 1e4, rng.random(k) * 1e4
    sig = 20 * 20 ** rng.random(k)
    c = rng.integers(0, k, n)
    return cx[c] + sig[c] * rng.standard_normal(n), cy[c] + sig[c] * rng.standard_normal(n)


def _check(gcore, xs, ys, form, order=8, opening=1.5, targets=1024, tol=TOL):
    kick, alpha = acc.many_body_kick(pkg, gcore, xs, ys, form=form, order=order, opening=opening)
    tg = acc.sample_targets(xs, ys, targets)
    ref = acc.direct_kick(xs, ys, np.full(len(xs), -30.0 * alpha), tg)
    r = acc.rms(kick, ref, tg)
    assert r <= tol, "%s order %d: RMS %.3g > %.3g" % (form, order, r, tol)
    return r


@pytest.mark.parametrize("n", [3000, 40000])
def test_gpu_tc_fmm_uniform_rms(gcore, n):
    xs, ys = _uniform(n, 3)
    _check(gcore, xs, ys, "bf16x3")


def test_gpu_tc_fmm_clustered_rms(gcore):
    xs, ys = _clusters(60000, 5)
    _check(gcore, xs, ys, "bf16x3")


def test_gpu_tc_fmm_coincident_and_nan_nodes(gcore):
    """Exact duplicates (the hashed jiggle in the FP32 near field) and nodes
    whose position becomes NaN after initialisation (d3 places NaN starting
    positions itself; later NaNs get no force and exert none) do not disturb
    the other nodes' kicks."""
    xs, ys = _uniform(20000, 9)
    xs[1::97] = xs[0:-1:97][: len(xs[1::97])]
    ys[1::97] = ys[0:-1:97][: len(ys[1::97])]
    n = len(xs)
    nodes = pkg.Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=gcore)
    sim.force("charge", pkg.forceManyBody())
    sim.precision("fast", order=8, opening=1.5, form="bf16x3")
    nodes.x[5::1009] = np.nan
    ok = ~np.isnan(np.asarray(nodes.x))
    sim.tick()
    alpha = sim.alpha()
    kick = np.stack([np.asarray(nodes.vx), np.asarray(nodes.vy)], 1) / 0.6
    sim.close()
    assert np.all(kick[~ok] == 0)
    xv, yv = xs[ok], ys[ok]
    tg = acc.sample_targets(xv, yv, 512)
    ref = acc.direct_kick(xv, yv, np.full(len(xv), -30.0 * alpha), tg)
    assert acc.rms(kick[ok], ref, tg) <= TOL


def test_gpu_tc_fmm_order_controls_error(gcore):
    """Error falls with the expansion order: order 4 is coarser than 8, and
    order 12 is at least as close as 8."""
    xs, ys = _uniform(20000, 11)
    r4 = _check(gcore, xs, ys, "bf16x3", order=4, tol=1e-2)
    r8 = _check(gcore, xs, ys, "bf16x3", order=8)
    r12 = _check(gcore, xs, ys, "bf16x3", order=12)
    assert r4 > r8 and r12 <= r8 * 1.5


def test_gpu_tc_fmm_within_plain_fmm_error(gcore):
    """On the same layout the tensor-core form's error stays within a few
    times the reference FMM's (the FP64 plain form at order 8)."""
    xs, ys = _uniform(30000, 13)
    rp = _check(gcore, xs, ys, "plain")
    rt = _check(gcore, xs, ys, "bf16x3")
    assert rt <= max(5 * rp, 2e-6)


def test_gpu_tc_form_center_tree_sums(gcore):
    """With a many-body force in the tensor-core form, the center force's sums
    take the tree order (chunk sums, then one reduction) instead of the
    sequential order: the shift still equals the exact mean to FP64 rounding.
    A zero-strength many-body force leaves the velocities at zero, so the tick
    moves every node by exactly the center's shift (simple.zig:14-31)."""
    n = 100000
    xs, ys = _uniform(n, 21)
    nodes = pkg.Nodes(n, x=xs.copy(), y=ys.copy(), vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=gcore)
    sim.force("charge", pkg.forceManyBody().strength(0))
    sim.force("center", pkg.forceCenter(1234.5, -678.25))
    sim.precision("fast", order=8, opening=1.5, form="bf16x3")
    sim.tick()
    x1, y1 = np.asarray(nodes.x).copy(), np.asarray(nodes.y).copy()
    sim.close()
    import math
    sx = math.fsum(xs) / n - 1234.5
    sy = math.fsum(ys) / n + 678.25
    assert np.max(np.abs((xs - sx) - x1)) < 1e-9
    assert np.max(np.abs((ys - sy) - y1)) < 1e-9
