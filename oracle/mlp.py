"""CPU oracle of the learned-MAC network (numpy).

TEST INFRASTRUCTURE ONLY: checks the device MLP kernels (tree_b200/csrc/mlp.cu)
forward values and gradients.  The reference has no learned part; this oracle
restates the network the device trains: 16 -> 64 -> 64 -> 1 with ReLU, the
first two layers on BF16 tensor-core operands with FP32 accumulation, the last
layer in FP32, and the pinball (quantile) loss.

`bf16_emulation=True` rounds exactly the operands the device feeds to its BF16
mma instructions, so device and oracle agree to FP32 summation-order error.
"""
import numpy as np

N_IN, N_H = 16, 64
# flat FP32 parameter layout shared with the device (tree_gpu.h)
SHAPES = [("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
          ("w3", (N_H,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(flat):
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(flat[o:o + k], dtype=np.float32).reshape(shp)
        o += k
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], np.float32).ravel() for name, _ in SHAPES])


def bf16(x):
    """Round FP32 to bfloat16 (round to nearest even) and back."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    return pack({
        "W1": rng.standard_normal((N_IN, N_H)) * np.sqrt(2.0 / N_IN),
        "b1": np.zeros(N_H), "W2": rng.standard_normal((N_H, N_H)) * np.sqrt(2.0 / N_H),
        "b2": np.zeros(N_H), "w3": rng.standard_normal(N_H) * np.sqrt(1.0 / N_H),
        "b3": np.zeros(1)})


def forward(flat, X, bf16_emulation=True):
    p = unpack(flat)
    r = bf16 if bf16_emulation else (lambda a: np.asarray(a, np.float32))
    X = np.asarray(X, np.float32)
    Z1 = r(X) @ r(p["W1"]) + p["b1"]
    H1 = np.maximum(Z1, 0)
    Z2 = r(H1) @ r(p["W2"]) + p["b2"]
    H2 = np.maximum(Z2, 0)
    y = H2 @ p["w3"] + p["b3"][0]
    return y.astype(np.float32), (X, Z1, H1, Z2, H2)


def loss_and_grad(flat, X, y, tau=0.9, bf16_emulation=True):
    """Mean pinball loss and its gradient w.r.t. the flat parameters."""
    p = unpack(flat)
    r = bf16 if bf16_emulation else (lambda a: np.asarray(a, np.float32))
    yhat, (X, Z1, H1, Z2, H2) = forward(flat, X, bf16_emulation)
    e = np.asarray(y, np.float32) - yhat
    n = len(X)
    loss = float(np.mean(np.maximum(tau * e, (tau - 1) * e)))
    g = np.where(e > 0, -tau, 1 - tau).astype(np.float32) / n
    dW3 = H2.T @ g
    db3 = np.array([g.sum()], np.float32)
    dZ2 = (g[:, None] * p["w3"][None, :]) * (Z2 > 0)
    dW2 = r(H1).T @ r(dZ2)
    db2 = dZ2.sum(0)
    dH1 = r(dZ2) @ r(p["W2"]).T
    dZ1 = dH1 * (Z1 > 0)
    dW1 = r(X).T @ r(dZ1)
    db1 = dZ1.sum(0)
    grads = pack({"W1": dW1, "b1": db1, "W2": dW2, "b2": db2, "w3": dW3, "b3": db3})
    return loss, grads


def adam_step(flat, grad, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (t counts from 1); returns new (flat, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1**t)
    vh = v / (1 - b2**t)
    return (flat - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32), m, v
