"""Device tensor-core MLP kernels against the CPU oracle (oracle/mlp.py)."""
import numpy as np
import pytest

from oracle import mlp
from tree_b200 import api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 31, 32, 100, 4096, 10007])
def test_device_gradient_matches_oracle(device_lib, n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, 16)).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    p = mlp.init_params(n)
    loss_d, g_d = api.mlp_grad(X, y, p, tau=0.9)
    loss_o, g_o = mlp.loss_and_grad(p, X, y, tau=0.9, bf16_emulation=True)
    assert loss_d == pytest.approx(loss_o, rel=1e-4, abs=1e-6)
    # same BF16 operands, FP32 sums in another order
    scale = np.abs(g_o).max()
    assert np.abs(g_d - g_o).max() <= 2e-4 * scale
    for name, sl in (("W1", slice(0, 1024)), ("W2", slice(1088, 5184)), ("w3", slice(5248, 5312))):
        a, b = g_d[sl], g_o[sl]
        assert np.linalg.norm(a - b) <= 1e-3 * (np.linalg.norm(b) + 1e-12), name


def test_device_inference_matches_oracle(device_lib):
    rng = np.random.default_rng(7)
    X = rng.standard_normal((3000, 16)).astype(np.float32) * 2 + 1
    p = mlp.init_params(9)
    mean = rng.standard_normal(16).astype(np.float32)
    inv_std = rng.uniform(0.5, 2.0, 16).astype(np.float32)
    stats = np.concatenate([mean, inv_std, np.full(16, -1e30), np.full(16, 1e30),
                            np.zeros(8)]).astype(np.float32)
    y_d = api.mlp_infer(X, p, stats)
    y_o, _ = mlp.forward(p, (X - mean) * inv_std, bf16_emulation=True)
    np.testing.assert_allclose(y_d, y_o, rtol=1e-4, atol=1e-4 * np.abs(y_o).max())


def test_device_training_step_follows_oracle_adam(device_lib):
    """A few device gradient + oracle Adam steps stay on the oracle's path."""
    rng = np.random.default_rng(3)
    X = rng.standard_normal((2048, 16)).astype(np.float32)
    y = (np.tanh(X[:, 0]) + 0.3 * X[:, 5]).astype(np.float32)
    p_d = mlp.init_params(4)
    p_o = p_d.copy()
    md = np.zeros_like(p_d); vd = np.zeros_like(p_d)
    mo = np.zeros_like(p_o); vo = np.zeros_like(p_o)
    for t in range(1, 6):
        _, gd = api.mlp_grad(X, y, p_d, 0.5)
        _, go = mlp.loss_and_grad(p_o, X, y, 0.5)
        p_d, md, vd = mlp.adam_step(p_d, gd, md, vd, t)
        p_o, mo, vo = mlp.adam_step(p_o, go, mo, vo, t)
    assert np.abs(p_d - p_o).max() <= 1e-4
