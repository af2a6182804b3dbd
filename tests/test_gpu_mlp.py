"""Warm-start network kernels: tensor-core forward and FP32 backward against
the FP64 restatement in mlp_ref.py (same BF16 roundings), and Adam training
reducing the error on a smooth synthetic map."""
import ctypes as C

import numpy as np
import pytest

import mlp_ref
from imex_sflow2d_v2_b200.solver import ImexMLP

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 12)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2],
                  np.tanh(x[:, 3] - x[:, 4]) + 0.1 * x[:, 11]], 1).astype(np.float32)
    return x, y


def test_forward_and_gradient_match_fp64_reference():
    net = ImexMLP(seed=3)
    x, y = _data(1000, 1)           # not a multiple of the 64-sample tile
    p = net.params()
    loss_ref, g_ref, y_ref = mlp_ref.loss_grad(p, x, y)
    y_gpu = net.predict(x)
    assert np.abs(y_gpu - y_ref).max() <= 2e-3 * np.abs(y_ref).max()
    loss, g = net.loss_grad(x, y)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err <= 5e-3, err
    # padded rows of W0 and columns of W3 never receive gradient
    o, _ = mlp_ref.OFF["W0"]
    assert not g[o + 12 * 64:o + 16 * 64].any()


def test_adam_training_reduces_error():
    import torch
    net = ImexMLP(seed=5)
    x, y = _data(1 << 15, 2)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    before = net.loss_grad(x[:4096], y[:4096])[0]
    losses = net.train(C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), x.shape[0],
                       epochs=20, batch=1024, lr=2e-3)
    after = net.loss_grad(x[:4096], y[:4096])[0]
    assert losses[-1] < losses[0] and after < 0.1 * before, (before, after, losses)
