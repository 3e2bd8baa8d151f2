"""CPU checks of the learned-MAC network oracle (oracle/mlp.py)."""
import numpy as np

from oracle import mlp


def test_pack_unpack_roundtrip():
    p = mlp.init_params(3)
    assert p.size == mlp.N_PARAMS == 5313
    np.testing.assert_array_equal(mlp.pack(mlp.unpack(p)), p)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, -2.5e-3, 3.0e38], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # exact tie -> even
    assert r[2] == np.float32(1.0 + 2**-7)
    rel = np.abs(r - x) / np.abs(x)
    assert np.all(rel <= 2**-8)  # half an ulp of an 8-bit significand


def test_gradient_matches_finite_differences():
    """Exact (FP32, no BF16) oracle gradient vs central differences of the loss
    with a smooth surrogate: use tau so the loss is linear away from kinks."""
    rng = np.random.default_rng(0)
    X = rng.standard_normal((64, 16)).astype(np.float32)
    y = rng.standard_normal(64).astype(np.float32) * 3
    p = mlp.init_params(1).astype(np.float64)
    loss, g = mlp.loss_and_grad(p.astype(np.float32), X, y, tau=0.8, bf16_emulation=False)
    idx = rng.choice(p.size, 40, replace=False)
    for i in idx:
        h = 1e-3
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = mlp.loss_and_grad(pp.astype(np.float32), X, y, 0.8, False)
        lm, _ = mlp.loss_and_grad(pm.astype(np.float32), X, y, 0.8, False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])) + 1e-4, (i, fd, g[i])


def test_adam_reduces_loss():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((512, 16)).astype(np.float32)
    y = (X[:, 0] * 2 - X[:, 3]).astype(np.float32)
    p = mlp.init_params(2)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    l0, _ = mlp.loss_and_grad(p, X, y, 0.5)
    for t in range(1, 201):
        _, g = mlp.loss_and_grad(p, X, y, 0.5)
        p, m, v = mlp.adam_step(p, g, m, v, t, lr=3e-3)
    l1, _ = mlp.loss_and_grad(p, X, y, 0.5)
    assert l1 < 0.5 * l0
