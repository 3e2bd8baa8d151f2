"""CPU checks of the walk's local (Taylor) expansion of far cells about a
target group's centre (tree_b200/csrc/local.cuh), built for the host from the
same source the device compiles.

The multipole series of a random cluster (net charge, dipole and trace-free
second to fourth moments about its centroid, as the upward pass stores them)
is evaluated in FP64 here; the expansion's coefficients must be its value and
derivatives at the group centre, and the expanded force at targets around the
centre must converge to the series' force as the fourth power of h/d.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "local_harness.cpp")
INC = os.path.join(ROOT, "tree_b200", "csrc")


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("local") / "local_harness.so")
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-std=c++17", "-ffp-contract=off",
                    "-I", INC, SRC, "-o", so], check=True)
    L = ctypes.CDLL(so)
    fp = ctypes.POINTER(ctypes.c_float)
    L.loc_coefs.argtypes = [ctypes.c_int, fp, fp, fp]
    L.loc_eval.argtypes = [fp, fp, fp]
    return L


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def coefs(lib, order, d0, m):
    d, dp = _f32(d0)
    mm, mp = _f32(m)
    c, cp = _f32(np.zeros(29))
    lib.loc_coefs(order, dp, mp, cp)
    return c.astype(np.float64)


def evaluate(lib, c, t):
    cc, cp = _f32(c)
    tt, tp = _f32(t)
    out, op = _f32(np.zeros(5))
    lib.loc_eval(cp, tp, op)
    return out.astype(np.float64)


# ---- the cluster and its trace-free moments (FP64) ----
def cluster(rng, n=40, a=1.0, bias=0.1):
    pos = rng.normal(size=(n, 3)) * a / 2
    q = np.where(rng.random(n) < 0.5 + bias, 1.0, -1.0)
    X = (pos).mean(0)  # expansion centre: the particles' centroid
    return pos - X, q


def detrace2(S):
    return S - np.trace(S) / 3 * np.eye(3)


def detrace3(T):
    V = np.einsum("iik->k", T)
    I = np.eye(3)
    return T - (np.einsum("ij,k->ijk", I, V) + np.einsum("ik,j->ijk", I, V) +
                np.einsum("jk,i->ijk", I, V)) / 5


def detrace4(H):
    I = np.eye(3)
    H2 = np.einsum("ijmm->ij", H)
    h0 = np.trace(H2)
    t1 = sum(np.einsum(s, I, H2) for s in ("ij,kl->ijkl", "ik,jl->ijkl", "il,jk->ijkl",
                                          "jk,il->ijkl", "jl,ik->ijkl", "kl,ij->ijkl"))
    t2 = (np.einsum("ij,kl->ijkl", I, I) + np.einsum("ik,jl->ijkl", I, I) +
          np.einsum("il,jk->ijkl", I, I))
    return H - t1 / 7 + t2 * h0 / 35


def moments(a, q):
    Q = q.sum()
    D = (q[:, None] * a).sum(0)
    S = detrace2(0.5 * np.einsum("n,ni,nj->ij", q, a, a))
    T = detrace3(np.einsum("n,ni,nj,nk->ijk", q, a, a, a))
    H = detrace4(np.einsum("n,ni,nj,nk,nl->ijkl", q, a, a, a, a))
    return Q, D, S, T, H


def pack(Q, D, S, T, H, q_ion):
    s = [S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[1, 2], S[2, 0]]
    idx3 = [(0, 0, 0), (1, 1, 1), (2, 2, 2), (0, 0, 1), (0, 0, 2), (0, 1, 1), (1, 1, 2),
            (0, 2, 2), (1, 2, 2), (0, 1, 2)]
    idx4 = [(0, 0, 0, 0), (0, 0, 0, 1), (0, 0, 0, 2), (0, 0, 1, 1), (0, 0, 1, 2),
            (0, 1, 1, 1), (0, 1, 1, 2), (1, 1, 1, 1), (1, 1, 1, 2), (0, 0, 2, 2),
            (0, 1, 2, 2), (1, 1, 2, 2)]
    return np.array([Q, *D, *s, *[T[i] for i in idx3], *[H[i] for i in idx4], q_ion])


def series(d, mom, upto=4):
    """The walk's multipole series phi(d) up to order `upto`."""
    Q, D, S, T, H = mom
    r = np.linalg.norm(d)
    phi = Q / r
    if upto >= 1:
        phi += D @ d / r**3
    if upto >= 2:
        phi += 3 * d @ S @ d / r**5
    if upto >= 3:
        phi += 2.5 * np.einsum("ijk,i,j,k->", T, d, d, d) / r**7
    if upto >= 4:
        phi += 4.375 * np.einsum("ijkl,i,j,k,l->", H, d, d, d, d) / r**9
    return phi


def fd_grad(f, x, h):
    g = np.zeros(3)
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        g[i] = (8 * (f(x + e) - f(x - e)) - (f(x + 2 * e) - f(x - 2 * e))) / (12 * h)
    return g


def derivatives(d0, mom, upto, k):
    """k-th derivative tensor of the series (orders to `upto`) at d0, exact
    (forward-mode automatic differentiation in FP64)."""
    import torch
    from torch.func import jacfwd
    Q, D, S, T, H = (torch.as_tensor(np.asarray(m, dtype=np.float64)) for m in mom)

    def phi(d):
        r = torch.linalg.norm(d)
        out = Q / r
        if upto >= 1:
            out = out + D @ d / r**3
        if upto >= 2:
            out = out + 3 * d @ S @ d / r**5
        if upto >= 3:
            out = out + 2.5 * torch.einsum("ijk,i,j,k->", T, d, d, d) / r**7
        if upto >= 4:
            out = out + 4.375 * torch.einsum("ijkl,i,j,k,l->", H, d, d, d, d) / r**9
        return out
    f = phi
    for _ in range(k):
        f = jacfwd(f)
    return f(torch.as_tensor(np.asarray(d0, dtype=np.float64))).numpy()


def unpack_L(c):
    import itertools
    Lxxxx, Lxxxy, Lxxyy, Lxyyy, Lyyyy, Lxxxz, Lxxyz, Lxyyz, Lyyyz = c[20:29]
    Lxxzz, Lxyzz, Lyyzz = -(Lxxxx + Lxxyy), -(Lxxxy + Lxyyy), -(Lxxyy + Lyyyy)
    Lxzzz, Lyzzz = -(Lxxxz + Lxyyz), -(Lxxyz + Lyyyz)
    vals = {(0, 0, 0, 0): Lxxxx, (0, 0, 0, 1): Lxxxy, (0, 0, 1, 1): Lxxyy, (0, 1, 1, 1): Lxyyy,
            (1, 1, 1, 1): Lyyyy, (0, 0, 0, 2): Lxxxz, (0, 0, 1, 2): Lxxyz, (0, 1, 1, 2): Lxyyz,
            (1, 1, 1, 2): Lyyyz, (0, 0, 2, 2): Lxxzz, (0, 1, 2, 2): Lxyzz, (1, 1, 2, 2): Lyyzz,
            (0, 2, 2, 2): Lxzzz, (1, 2, 2, 2): Lyzzz, (2, 2, 2, 2): -(Lxxzz + Lyyzz)}
    L = np.zeros((3, 3, 3, 3))
    for key, v in vals.items():
        for p in itertools.permutations(key):
            L[p] = v
    return L


def unpack_H(c):
    Hxx, Hyy, Hxy, Hxz, Hyz = c[4:9]
    return np.array([[Hxx, Hxy, Hxz], [Hxy, Hyy, Hyz], [Hxz, Hyz, -Hxx - Hyy]])


def unpack_K(c):
    Kxxx, Kyyy, Kxxy, Kxxz, Kxyy, Kyyz, Kxyz = c[9:16]
    K = np.zeros((3, 3, 3))
    vals = {(0, 0, 0): Kxxx, (1, 1, 1): Kyyy, (0, 0, 1): Kxxy, (0, 0, 2): Kxxz,
            (0, 1, 1): Kxyy, (1, 1, 2): Kyyz, (0, 1, 2): Kxyz,
            (0, 2, 2): -(Kxxx + Kxyy), (1, 2, 2): -(Kxxy + Kyyy), (2, 2, 2): -(Kxxz + Kyyz)}
    import itertools
    for key, v in vals.items():
        for p in itertools.permutations(key):
            K[p] = v
    return K


@pytest.mark.parametrize("order", [2, 3, 4])
def test_coefficients_are_the_series_derivatives(lib, order):
    rng = np.random.default_rng(11 + order)
    for trial in range(4):
        a, q = cluster(rng)
        mom = moments(a, q)
        q_ion = float((q > 0).sum())
        d0 = rng.normal(size=3)
        d0 *= (6.0 + 4 * trial) / np.linalg.norm(d0)
        c = coefs(lib, order, d0, pack(*mom, q_ion))
        r = np.linalg.norm(d0)
        f_all = lambda x: series(x, mom, order)
        # phi0 and g carry every order of the walk
        assert c[0] == pytest.approx(f_all(d0), rel=2e-5, abs=1e-6 * len(q) / r)
        g = derivatives(d0, mom, order, 1)
        np.testing.assert_allclose(c[1:4], g, rtol=0, atol=2e-5 * np.abs(g).max() + 1e-7 * len(q) / r**2)
        # H: every order; K: multipoles to T; L: multipoles to S
        Hs = derivatives(d0, mom, order, 2)
        np.testing.assert_allclose(unpack_H(c), Hs, rtol=0, atol=1e-4 * np.abs(Hs).max())
        Ks = derivatives(d0, mom, min(order, 3), 3)
        np.testing.assert_allclose(unpack_K(c), Ks, rtol=0, atol=1e-4 * np.abs(Ks).max())
        Ls = derivatives(d0, mom, 2, 4)
        np.testing.assert_allclose(unpack_L(c), Ls, rtol=0, atol=1e-4 * np.abs(Ls).max())
        # ion monopole part
        assert c[16] == pytest.approx(q_ion / r, rel=1e-5)
        np.testing.assert_allclose(c[17:20], -q_ion * d0 / r**3, rtol=1e-5)


def test_expanded_force_converges_as_fourth_power(lib):
    rng = np.random.default_rng(5)
    a, q = cluster(rng, n=60, bias=0.02)
    mom = moments(a, q)
    d0 = np.array([7.0, -3.0, 4.5])
    c = coefs(lib, 4, d0, pack(*mom, float((q > 0).sum())))
    r = np.linalg.norm(d0)
    errs = []
    for hr in (0.2, 0.1, 0.05):
        worst = 0.0
        for k in range(20):
            t = rng.normal(size=3)
            t *= hr * r / np.linalg.norm(t)
            out = evaluate(lib, c, t)
            f_ref = -fd_grad(lambda x: series(x, mom, 4), d0 + t, 1e-3 * r)
            phi_ref = series(d0 + t, mom, 4)
            worst = max(worst, np.linalg.norm(out[:3] - f_ref) / np.linalg.norm(f_ref))
            assert out[3] == pytest.approx(phi_ref, rel=0.05 * hr**2 + 1e-5)
        errs.append(worst)
    # (h/d)^4: halving h cuts the error about sixteenfold (at least eightfold)
    assert errs[0] > 8 * errs[1] > 64 * errs[2] * 0.5, errs
    assert errs[2] < 2e-4


def test_evaluation_is_the_taylor_polynomial(lib):
    rng = np.random.default_rng(9)
    for _ in range(20):
        c = rng.normal(size=29)
        t = rng.normal(size=3)
        out = evaluate(lib, c, t)
        c32 = c.astype(np.float32).astype(np.float64)
        H, K, L = unpack_H(c32), unpack_K(c32), unpack_L(c32)
        g = (c32[1:4] + H @ t + 0.5 * np.einsum("ijk,j,k->i", K, t, t) +
             np.einsum("ijkl,j,k,l->i", L, t, t, t) / 6)
        phi = (c32[0] + c32[1:4] @ t + 0.5 * t @ H @ t +
               np.einsum("ijk,i,j,k->", K, t, t, t) / 6 +
               np.einsum("ijkl,i,j,k,l->", L, t, t, t, t) / 24)
        scale = np.abs(c32).max() * (1 + np.abs(t).max()) ** 4
        np.testing.assert_allclose(out[:3], -g, atol=1e-5 * scale)
        assert out[3] == pytest.approx(phi, abs=1e-5 * scale)
        assert out[4] == pytest.approx(c32[16] + c32[17:20] @ t, abs=1e-5 * scale)


@pytest.mark.parametrize("which", ["Q", "D", "S", "T", "H"])
def test_each_multipole_order_alone(lib, which):
    """One moment at a time (the others zero), so that an error in any one
    order's coefficients cannot hide behind the larger low orders."""
    import itertools
    import math
    rng = np.random.default_rng({"Q": 1, "D": 2, "S": 3, "T": 4, "H": 5}[which])

    def sym(rank):
        a = rng.normal(size=(3,) * rank)
        return sum(np.transpose(a, p) for p in itertools.permutations(range(rank))) / math.factorial(rank)
    Q, D = 0.0, np.zeros(3)
    S, T, H = np.zeros((3, 3)), np.zeros((3, 3, 3)), np.zeros((3, 3, 3, 3))
    if which == "Q":
        Q = 1.5
    elif which == "D":
        D = rng.normal(size=3)
    elif which == "S":
        S = detrace2(sym(2))
    elif which == "T":
        T = detrace3(sym(3))
    else:
        H = detrace4(sym(4))
    mom = (Q, D, S, T, H)
    for trial in range(3):
        d0 = rng.normal(size=3)
        d0 *= 3.0 / np.linalg.norm(d0)
        c = coefs(lib, 4, d0, pack(*mom, 0.0))
        for k, got, upto in ((0, c[0], 4), (1, c[1:4], 4), (2, unpack_H(c), 4),
                             (3, unpack_K(c), 3), (4, unpack_L(c), 2)):
            want = derivatives(d0, mom, upto, k)
            scale = np.abs(derivatives(d0, mom, 4, k)).max()
            np.testing.assert_allclose(got, want, rtol=0, atol=3e-6 * scale,
                                       err_msg=f"{which} derivative {k}")
