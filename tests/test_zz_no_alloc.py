"""The allocation-free many-body entry point against force_run.

d3_many_body_exact_noalloc serves callers that cannot let a library allocate
device memory (engines that own all GPU memory, latency-bound loops where
cudaMalloc would synchronise): it runs the exact many-body force on the
caller's device buffers with its scratch in a static device array. Here the
test itself allocates the buffers (with torch) and compares the entry point's
output with the existing path (force_run of a many-body force through the
simulation ABI): bit for bit, the exact-mode tolerance, on two calls in a row.
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

import helpers as H

C = H.C
pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.d3_many_body_exact_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_uint32] + [ctypes.c_double] * 4 + [
        ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p]
    return fn


def _nodes(n, seed):
    rnd = H.pkg.d3_lcg(seed)
    x = np.array([(rnd() - 0.5) * 800 for _ in range(n)])
    y = np.array([(rnd() - 0.5) * 800 for _ in range(n)])
    for k in range(0, n, 97):  # coincident pairs: the jiggle path draws
        x[k + 1 if k + 1 < n else k] = x[k]
        y[k + 1 if k + 1 < n else k] = y[k]
    vx = np.array([(rnd() - 0.5) for _ in range(n)])
    vy = np.array([(rnd() - 0.5) for _ in range(n)])
    strength = np.array([-30.0 - (k % 7) for k in range(n)])
    return x, y, vx, vy, strength


def _force_run(gcore, x, y, vx, vy, strength, alpha, lcg):
    """The existing path: one exact many-body force_run on a simulation."""
    n = len(x)
    h = gcore.sim_create()
    try:
        assert gcore.sim_set_node_count(h, n) >= 0
        gcore.sim_set_sync(h, C.SYNC_EXPLICIT)
        for w, arr in ((C.PTR_X, x), (C.PTR_Y, y), (C.PTR_VX, vx), (C.PTR_VY, vy)):
            gcore.f64_view(gcore.sim_ptr(h, w), n)[:] = arr
        gcore.u8_view(gcore.sim_ptr(h, C.PTR_FIXED), n)[:] = 0
        fh = gcore.force_create(h, C.MANY_BODY)
        gcore.f64_view(gcore.force_ptr(h, fh, C.F0), n)[:] = strength
        gcore.force_set_scalar(h, fh, C.THETA2, 0.81)
        gcore.force_set_scalar(h, fh, C.DISTANCE_MIN2, 1.0)
        gcore.force_set_scalar(h, fh, C.DISTANCE_MAX2, float("inf"))
        assert gcore.sim_set_lcg(h, lcg) == 0
        assert gcore.sim_sync_in(h) == 0
        assert gcore.force_run(h, fh, alpha) == 0
        assert gcore.sim_sync_out(h) == 0
        out_vx = gcore.f64_view(gcore.sim_ptr(h, C.PTR_VX), n).copy()
        out_vy = gcore.f64_view(gcore.sim_ptr(h, C.PTR_VY), n).copy()
        return out_vx, out_vy, gcore.sim_get_lcg(h)
    finally:
        gcore.sim_destroy(h)


def test_no_alloc_many_body_matches_force_run(gcore):
    import torch

    fn = _bind(gcore.lib)
    n = 6000
    x, y, vx, vy, strength = _nodes(n, 7)
    dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    tx, ty, tvx, tvy, ts = dev(x), dev(y), dev(vx), dev(vy), dev(strength)
    lcg_ref, lcg = 1, ctypes.c_uint32(1)
    ref_vx, ref_vy = vx, vy
    for call, alpha in enumerate((0.99, 0.97)):
        ref_vx, ref_vy, lcg_ref = _force_run(gcore, x, y, ref_vx, ref_vy, strength, alpha, lcg_ref)
        torch.cuda.synchronize()
        rc = fn(tx.data_ptr(), ty.data_ptr(), tvx.data_ptr(), tvy.data_ptr(), ts.data_ptr(), n,
                0.81, 1.0, float("inf"), alpha, ctypes.byref(lcg), None)
        assert rc == 0, "call %d: status %d" % (call, rc)
        got_vx, got_vy = tvx.cpu().numpy(), tvy.cpu().numpy()
        assert np.array_equal(got_vx.view(np.uint64), ref_vx.view(np.uint64)), "call %d: vx" % call
        assert np.array_equal(got_vy.view(np.uint64), ref_vy.view(np.uint64)), "call %d: vy" % call
        assert lcg.value == lcg_ref, "call %d: random stream position" % call
    assert lcg_ref != 1  # the coincident pairs drew from the stream


def test_no_alloc_many_body_matches_oracle(ocore, gcore):
    """The entry point against the CPU oracle's force_run directly (the
    oracle restates many_body.zig), bit for bit, on two calls in a row."""
    import torch

    fn = _bind(gcore.lib)
    n = 3000
    x, y, vx, vy, strength = _nodes(n, 11)
    dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    tx, ty, tvx, tvy, ts = dev(x), dev(y), dev(vx), dev(vy), dev(strength)
    lcg_ref, lcg = 1, ctypes.c_uint32(1)
    ref_vx, ref_vy = vx, vy
    for call, alpha in enumerate((0.5, 0.25)):
        ref_vx, ref_vy, lcg_ref = _force_run(ocore, x, y, ref_vx, ref_vy, strength, alpha, lcg_ref)
        rc = fn(tx.data_ptr(), ty.data_ptr(), tvx.data_ptr(), tvy.data_ptr(), ts.data_ptr(), n,
                0.81, 1.0, float("inf"), alpha, ctypes.byref(lcg), None)
        assert rc == 0, "call %d: status %d" % (call, rc)
        got_vx, got_vy = tvx.cpu().numpy(), tvy.cpu().numpy()
        assert np.array_equal(got_vx.view(np.uint64), ref_vx.view(np.uint64)), "call %d: vx" % call
        assert np.array_equal(got_vy.view(np.uint64), ref_vy.view(np.uint64)), "call %d: vy" % call
        assert lcg.value == lcg_ref, "call %d: random stream position" % call


def test_no_alloc_tree_overflow_is_reported_and_harmless(gcore):
    """Points whose tree needs more cells than the static array holds
    (clustered pairs: about 7.3n cells against 4n + 1024, checked on the
    oracle in test_oracle.py) return D3_ARENA_FULL with vx, vy and the random
    stream untouched, and the next call on ordinary points is correct."""
    import torch

    fn = _bind(gcore.lib)
    n = 8192
    x, y = H.clustered_pairs(n, 3)
    vx = np.linspace(-1, 1, n)
    dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    tx, ty, tvx, tvy, ts = dev(x), dev(y), dev(vx), dev(-vx), dev(np.full(n, -30.0))
    lcg = ctypes.c_uint32(12345)
    rc = fn(tx.data_ptr(), ty.data_ptr(), tvx.data_ptr(), tvy.data_ptr(), ts.data_ptr(), n,
            0.81, 1.0, float("inf"), 1.0, ctypes.byref(lcg), None)
    assert rc == C.ARENA_FULL
    assert np.array_equal(tvx.cpu().numpy().view(np.uint64), vx.view(np.uint64))
    assert np.array_equal(tvy.cpu().numpy().view(np.uint64), (-vx).view(np.uint64))
    assert lcg.value == 12345
    test_no_alloc_many_body_matches_force_run(gcore)


def test_no_alloc_rejects_too_many_nodes(gcore):
    fn = _bind(gcore.lib)
    lcg = ctypes.c_uint32(1)
    rc = fn(None, None, None, None, None, 8193, 0.81, 1.0, float("inf"), 1.0, ctypes.byref(lcg),
            None)
    assert rc == C.BAD_ARGUMENT
