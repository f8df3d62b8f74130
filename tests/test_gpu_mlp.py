"""The warm-start MLP's tcgen05 BF16 kernels against the CPU reference (GPU).

Forward outputs and gradients are compared with the float64 restatement in
oracle/mlp_ref.py, once with BF16 rounding at the points where the GPU keeps
BF16 tensors (tight: only FP32 accumulation order and rare BF16 ties differ)
and once exact (loose: the BF16 approximation error itself).
"""
import numpy as np
import pytest

import mlp_ref
from dgbgk.warmstart import MLP
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def draw(rng, n, n_in, n_out):
    x = rng.uniform(-1, 1, (n, n_in)).astype(np.float32)
    t = (0.5 * np.sin(np.arange(n_out)[None, :] * 0.01 + 3 * x[:, :1]) + 0.1 * x[:, 1:2]).astype(np.float32)
    return x, t


@pytest.mark.parametrize("width,depth,n_out,batch", [(512, 1, 256, 256), (256, 2, 128, 384), (128, 3, 384, 128)])
def test_forward_matches_reference(width, depth, n_out, batch):
    # K = 64 (input layer), K = width (8 K-blocks wrap the 4-stage ring
    # twice at 512), N tiles of 128 and of 64 (the input layer's dW)
    m = MLP(3, width, depth, n_out, batch, seed=7)
    rng = np.random.default_rng(1)
    x, _ = draw(rng, batch + 37, 3, n_out)   # a ragged last chunk
    y = m.forward(x)
    p = m.get_params()
    ref, _ = mlp_ref.forward(p, x, 3, width, depth, n_out, bf16_points=True)
    exact, _ = mlp_ref.forward(p, x, 3, width, depth, n_out, bf16_points=False)
    assert np.isfinite(y).all()
    assert rel_l2(y, ref) <= 5e-3
    assert rel_l2(y, exact) <= 3e-2
    m.close()


def test_forward_single_layer_gemm_is_exact_to_fp32():
    # one hidden layer and inputs that are exactly representable in BF16:
    # the first GEMM's products are exact, so the GPU's hidden layer agrees
    # with the BF16-point reference to FP32 rounding before tanh
    m = MLP(3, 128, 1, 128, 128, seed=3)
    p = mlp_ref.bf16(m.get_params()).astype(np.float32)
    m.set_params(p)
    x = mlp_ref.bf16(np.random.default_rng(2).uniform(-1, 1, (128, 3))).astype(np.float32)
    y = m.forward(x)
    ref, _ = mlp_ref.forward(p, x, 3, 128, 1, 128, bf16_points=True)
    assert rel_l2(y, ref) <= 2e-3


@pytest.mark.parametrize("width,depth,n_out,batch", [(256, 2, 128, 384), (512, 4, 1024, 256)])
def test_gradient_matches_reference(width, depth, n_out, batch):
    m = MLP(3, width, depth, n_out, batch, seed=11)
    x, t = draw(np.random.default_rng(5), batch, 3, n_out)
    loss, g = m.gradient(x, t)
    p = m.get_params()
    rl, rg = mlp_ref.loss_and_grad(p, x, t, 3, width, depth, n_out, bf16_points=True)
    el, eg = mlp_ref.loss_and_grad(p, x, t, 3, width, depth, n_out, bf16_points=False)
    assert abs(loss - rl) <= 1e-3 * rl
    assert rel_l2(g, rg) <= 2e-2
    assert rel_l2(g, eg) <= 5e-2
    # per layer, so that a wrong layer cannot hide behind a large one
    o = 0
    for (no, ni, live) in mlp_ref.shapes(3, width, depth, n_out):
        gw, rw = g[o:o + no * ni].reshape(no, ni)[:, :live], rg[o:o + no * ni].reshape(no, ni)[:, :live]
        assert rel_l2(gw, rw) <= 3e-2
        o += no * ni
        assert rel_l2(g[o:o + no], rg[o:o + no]) <= 3e-2
        o += no
    m.close()


def test_training_reduces_loss():
    m = MLP(3, 256, 2, 256, 128, seed=2)
    x, t = draw(np.random.default_rng(9), 512, 3, 256)
    m.set_data(x, t)
    y0 = m.forward(x)
    hist = m.train(300, lr=2e-3, seed=4)
    y1 = m.forward(x)
    assert np.isfinite(hist).all()
    e0 = np.mean((y0 - t) ** 2)
    e1 = np.mean((y1 - t) ** 2)
    assert e1 < 0.2 * e0
    assert hist[-20:].mean() < 0.3 * hist[:5].mean()
    m.close()


def test_params_round_trip():
    m = MLP(3, 128, 1, 128, 128, seed=1)
    p = m.get_params()
    q = (p * 0.5).astype(np.float32)
    m.set_params(q)
    assert np.array_equal(m.get_params(), q)
    m.close()
