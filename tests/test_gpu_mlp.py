"""The learned correction's network on the B200: the training kernel's
gradients against a CPU restatement of the same network in FP64 (the same
bf16-rounded weights and activations), the tensor-core inference against the
CUDA-core forward pass, and a short training run that lowers the loss."""

import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

IN, HID, OUT = 12, 64, 2
P_W1 = 0
P_B1 = P_W1 + HID * IN
P_W2 = P_B1 + HID
P_B2 = P_W2 + HID * HID
P_W3 = P_B2 + HID
P_B3 = P_W3 + OUT * HID
NP = P_B3 + OUT


def _bind(lib):
    f = ctypes.POINTER(ctypes.c_float)
    lib.d3_mlp_grad.restype = ctypes.c_int32
    lib.d3_mlp_grad.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, f, f, f]
    lib.d3_mlp_infer.restype = ctypes.c_int32
    lib.d3_mlp_infer.argtypes = [ctypes.c_void_p, ctypes.c_uint32, f, ctypes.c_void_p,
                                 ctypes.c_uint32]
    lib.d3_mlp_train.restype = ctypes.c_int32
    lib.d3_mlp_train.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, f, f]
    return lib


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def bf16(a):
    """Round to bf16 (nearest even), returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _gelu(z):
    from scipy.special import erf
    return 0.5 * z * (1 + erf(z / np.sqrt(2)))


def _gelu_d(z):
    from scipy.special import erf
    return 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def cpu_grad(x, y, p):
    """The network and its loss gradient in FP64 with the GPU's roundings
    (weights and activations to bf16)."""
    W1 = bf16(p[P_W1:P_B1]).reshape(HID, IN)
    b1 = p[P_B1:P_W2].astype(np.float64)
    W2 = bf16(p[P_W2:P_B2]).reshape(HID, HID)
    b2 = p[P_B2:P_W3].astype(np.float64)
    W3 = bf16(p[P_W3:P_B3]).reshape(OUT, HID)
    b3 = p[P_B3:].astype(np.float64)
    xb = bf16(x)
    z1 = xb @ W1.T + b1
    a1 = bf16(_gelu(z1))
    z2 = a1 @ W2.T + b2
    a2 = bf16(_gelu(z2))
    yy = a2 @ W3.T + b3
    n = len(x)
    d = yy - y
    loss = (d * d).sum() / n
    dy = 2 * d / n
    dz2 = (dy @ W3) * _gelu_d(z2)
    dz1 = (dz2 @ W2) * _gelu_d(z1)
    g = np.zeros(NP)
    g[P_W1:P_B1] = (dz1.T @ xb).ravel()
    g[P_B1:P_W2] = dz1.sum(0)
    g[P_W2:P_B2] = (dz2.T @ a1).ravel()
    g[P_B2:P_W3] = dz2.sum(0)
    g[P_W3:P_B3] = (dy.T @ a2).ravel()
    g[P_B3:] = dy.sum(0)
    return g, loss, yy


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, IN)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0]) + 0.3 * x[:, 1] * x[:, 2], np.tanh(x[:, 3] - x[:, 4])], 1)
    p = np.zeros(NP, np.float32)
    p[P_W1:P_B1] = rng.standard_normal(HID * IN) * np.sqrt(2 / IN)
    p[P_W2:P_B2] = rng.standard_normal(HID * HID) * np.sqrt(2 / HID)
    p[P_W3:P_B3] = rng.standard_normal(OUT * HID) * np.sqrt(1 / HID)
    p[P_B1:P_W2] = 0.01
    return x, y.astype(np.float32), p


def test_gpu_mlp_gradients_match_cpu(gcore):
    import torch

    lib = _bind(gcore.lib)
    x, y, p = _data(1000, 1)
    tx, ty = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    g = np.zeros(NP, np.float32)
    loss = np.zeros(1, np.float32)
    assert lib.d3_mlp_grad(tx.data_ptr(), ty.data_ptr(), len(x), _fp(p), _fp(g), _fp(loss)) == 0
    gr, lr, _ = cpu_grad(x.astype(np.float64), y.astype(np.float64), p)
    assert abs(loss[0] - lr) <= 1e-4 * lr + 1e-6
    # FP32 sums of bf16 products: relative error per block of the gradient
    for a, b in ((P_W1, P_B1), (P_B1, P_W2), (P_W2, P_B2), (P_B2, P_W3), (P_W3, P_B3), (P_B3, NP)):
        err = np.linalg.norm(g[a:b] - gr[a:b]) / (np.linalg.norm(gr[a:b]) + 1e-12)
        assert err < 2e-3, (a, b, err)


def test_gpu_mlp_tensor_core_inference_matches(gcore):
    import torch

    lib = _bind(gcore.lib)
    x, _, p = _data(1000, 2)
    tx = torch.from_numpy(x).cuda()
    y_tc = torch.zeros(len(x), OUT, dtype=torch.float32, device="cuda")
    y_cc = torch.zeros_like(y_tc)
    assert lib.d3_mlp_infer(tx.data_ptr(), len(x), _fp(p), y_tc.data_ptr(), 1) == 0
    assert lib.d3_mlp_infer(tx.data_ptr(), len(x), _fp(p), y_cc.data_ptr(), 0) == 0
    a, b = y_tc.cpu().numpy(), y_cc.cpu().numpy()
    _, _, yr = cpu_grad(x.astype(np.float64), np.zeros((len(x), OUT)), p)
    # both hold bf16 activations: they agree to the bf16 rounding of a few
    # activations that land on a rounding boundary
    assert np.abs(a - b).max() <= 2e-2 * np.abs(b).max()
    assert np.abs(b - yr).max() <= 1e-2 * np.abs(yr).max()


def test_gpu_mlp_training_lowers_the_loss(gcore):
    import torch

    lib = _bind(gcore.lib)
    x, y, p = _data(20000, 3)
    tx, ty = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    steps = 300
    losses = np.zeros(steps, np.float32)
    assert lib.d3_mlp_train(tx.data_ptr(), ty.data_ptr(), len(x), 1024, steps, 3e-3, _fp(p),
                            _fp(losses)) == 0
    assert losses[-20:].mean() < 0.3 * losses[:5].mean(), (losses[:5], losses[-20:])
