"""Batched fast mode on the B200 (no reference counterpart): the per-graph
many-body kick against an FP64 direct sum (the fast mode's judge,
test/fast/error-test.js:44-70) on 256 sampled targets per graph; results
independent of the launch shape and of the CUDA-graph capture (the
reference's determinism contract: results do not depend on how the work is
split, src/core/pool.zig:7-10); and the ticks move the layout."""

import importlib

import numpy as np
import pytest

import helpers as H

B = importlib.import_module("d3-force-wasm_b200.batch")
pytestmark = pytest.mark.gpu


def _graphs(k=48, seed=2, nmax=4096):
    return B.batch_workload(k, seed=seed, nmax=nmax)


def test_gpu_batch_many_body_rms_per_graph(gcore):
    graphs = _graphs()
    b = B.Batch(gcore, graphs)
    try:
        kick, alpha = b.kick()
        rms = B.graph_rms(b, kick, alpha, range(len(graphs)))
        print("per-graph RMS: median %.3g max %.3g" % (np.median(rms), rms.max()))
        assert rms.max() < 1e-4
    finally:
        b.close()


def _state(b):
    return np.concatenate([a.view(np.uint32) for a in b.read()])


def test_gpu_batch_results_independent_of_launch_shape_and_graph(gcore):
    graphs = _graphs(24, seed=5)
    out = []
    for shape, graph in (((256, 1, 16), False), ((1024, 1, 16), True), ((512, 2, 16), True)):
        b = B.Batch(gcore, graphs)
        try:
            b.set_shape(*shape)
            b.run(4, graph=graph)
            b.run(6, graph=graph)
            out.append(_state(b))
        finally:
            b.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


def test_gpu_batch_ticks_move_and_autotune_picks_a_shape(gcore):
    graphs = _graphs(32, seed=7)
    b = B.Batch(gcore, graphs)
    try:
        choice = b.autotune(ticks=2)
        assert choice["threads"] in (256, 512, 1024) and choice["ms_per_tick"] > 0
        x0 = b.x0.copy()
        ms = b.run(20, graph=True)
        x, y, vx, vy = b.read()
        assert ms > 0 and np.all(np.isfinite(x)) and np.all(np.isfinite(vx))
        assert np.abs(x - x0).max() > 1e-3
    finally:
        b.close()


def _restated_tick(n, src, tgt, x, y):
    """One batched tick of one graph in FP64 (numpy), from zero velocity:
    the many-body force as a direct sum (distanceMin 1), the Jacobi link
    (distance 30, strength 1 / min(degree), bias degree(source) / (degree(
    source) + degree(target)), from the snapshot x + v), the Jacobi collide
    (radius 3 each, an even share of each overlap, from the snapshot after the
    link), then v *= 0.6 and x += v (link_fast.zig, grid.zig, simple.zig)."""
    alpha = 1 - (1 - 0.001 ** (1 / 300))
    vx = np.zeros(n)
    vy = np.zeros(n)
    dx = x[None, :] - x[:, None]
    dy = y[None, :] - y[:, None]
    l = dx * dx + dy * dy
    l = np.where(l < 1, np.sqrt(l), l)
    w = np.where(l > 0, -30.0 * alpha / np.where(l > 0, l, 1), 0)
    vx += (dx * w).sum(1)
    vy += (dy * w).sum(1)
    deg = np.bincount(src, minlength=n) + np.bincount(tgt, minlength=n)
    px, py = x + vx, y + vy
    dvx, dvy = np.zeros(n), np.zeros(n)
    for s_, t_ in zip(src, tgt):
        ex, ey = px[t_] - px[s_], py[t_] - py[s_]
        ll = np.hypot(ex, ey)
        f = (ll - 30) / ll * alpha / min(deg[s_], deg[t_])
        b = deg[s_] / (deg[s_] + deg[t_])
        dvx[t_] -= ex * f * b
        dvy[t_] -= ey * f * b
        dvx[s_] += ex * f * (1 - b)
        dvy[s_] += ey * f * (1 - b)
    vx += dvx
    vy += dvy
    px, py = x + vx, y + vy
    cx = px[:, None] - px[None, :]
    cy = py[:, None] - py[None, :]
    d2 = cx * cx + cy * cy
    hit = (d2 < 36) & (d2 > 0)
    ll = np.sqrt(np.where(hit, d2, 1))
    push = np.where(hit, (6 - ll) / ll * 0.5, 0)
    vx += (cx * push).sum(1)
    vy += (cy * push).sum(1)
    vx *= 0.6
    vy *= 0.6
    return x + vx, y + vy, vx, vy


def test_gpu_batch_tick_matches_fp64_restatement(gcore):
    """One tick of small graphs, their nodes packed so that collisions occur,
    against the FP64 restatement: the FP32 tick agrees to 1e-4 of the largest
    velocity (the FMM's own error is about 1e-6)."""
    rng = np.random.default_rng(11)
    graphs, pos = [], []
    for n in (80, 150, 300, 600):
        src = rng.integers(0, n, 2 * n)
        tgt = (src + 1 + rng.integers(0, n - 1, 2 * n)) % n
        graphs.append((n, src.astype(np.uint32), tgt.astype(np.uint32)))
        side = 2.5 * np.sqrt(n)  # dense: many pairs closer than 6
        pos.append((rng.random(n) * side, rng.random(n) * side))
    b = B.Batch(gcore, graphs, positions=pos)
    try:
        b.run(1, graph=False)
        x, y, vx, vy = b.read()
    finally:
        b.close()
    o = 0
    for (n, src, tgt), (px, py) in zip(graphs, pos):
        px32 = px.astype(np.float32).astype(np.float64)
        py32 = py.astype(np.float32).astype(np.float64)
        rx, ry, rvx, rvy = _restated_tick(n, src.astype(np.int64), tgt.astype(np.int64), px32, py32)
        scale = max(np.abs(rvx).max(), np.abs(rvy).max())
        assert np.abs(vx[o:o + n] - rvx).max() <= 1e-4 * scale, n
        assert np.abs(vy[o:o + n] - rvy).max() <= 1e-4 * scale, n
        o += n
