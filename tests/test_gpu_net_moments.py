"""Net-charge moments of the combined tree (mixed path) against their
definitions, summed in numpy from the sorted particles (B200).

Every twig's record holds its count n, centroid X, net charge Q, ion count and
the moments D = sum q a, S = 1/2 sum q a a^T, T = sum q a a a and H = sum q a a
a a of a = x - X.  The device computes twigs of up to 2,048 particles by
direct sums (one thread, or one warp above 64 particles) and the larger ones
from their children by the parallel-axis rules, leaf children as point
charges; both must match the definition to rounding.
"""
import numpy as np
import pytest

from tree_b200 import api

pytestmark = pytest.mark.gpu

T_IDX = [(0, 0, 0), (1, 1, 1), (2, 2, 2), (0, 0, 1), (0, 0, 2), (0, 1, 1), (1, 1, 2),
         (0, 2, 2), (1, 2, 2), (0, 1, 2)]
H_IDX = [(0, 0, 0, 0), (1, 1, 1, 1), (2, 2, 2, 2), (0, 0, 0, 1), (0, 0, 0, 2), (0, 1, 1, 1),
         (1, 1, 1, 2), (0, 2, 2, 2), (1, 2, 2, 2), (0, 0, 1, 1), (0, 0, 2, 2), (1, 1, 2, 2),
         (0, 0, 1, 2), (0, 1, 1, 2), (0, 1, 2, 2)]
S_IDX = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]


def _cloud(n_half, seed):
    """A Gaussian cloud of electrons near their ions plus a few far outliers
    (lone particles in big cells: leaf children of the large twigs)."""
    rng = np.random.default_rng(seed)
    xi = rng.normal(0.0, 50.0, (n_half, 3))
    xe = xi + rng.normal(0.0, 0.5, (n_half, 3))
    xe[:6] = rng.uniform(-3000.0, 3000.0, (6, 3))
    xi[:3] = rng.uniform(-3000.0, 3000.0, (3, 3))
    return xe, xi


def _reference(p):
    """Record of one twig from its particles p (k, 4): n, X, moments[38]."""
    X = p[:, :3].mean(0)
    a = p[:, :3] - X
    q = np.where(p[:, 3] > 0.5, 1.0, -1.0)
    rec = np.zeros(38)
    rec[0] = len(p)
    rec[1] = q.sum()
    rec[2:5] = (q[:, None] * a).sum(0)
    rec[5] = p[:, 3].sum()
    rec[6:12] = [0.5 * np.sum(q * a[:, i] * a[:, j]) for i, j in S_IDX]
    rec[12:22] = [np.sum(q * a[:, i] * a[:, j] * a[:, k]) for i, j, k in T_IDX]
    rec[22:37] = [np.sum(q * a[:, i] * a[:, j] * a[:, k] * a[:, l]) for i, j, k, l in H_IDX]
    r = np.linalg.norm(a, axis=1)
    # per-component scale: the sum of the magnitudes of the terms of its order
    scale = np.zeros(38)
    scale[2:5] = r.sum()
    scale[6:12] = (r ** 2).sum()
    scale[12:22] = (r ** 3).sum()
    scale[22:37] = (r ** 4).sum()
    return X, rec, scale, np.abs(p[:, :3]).max()


@pytest.mark.parametrize("n_half", [40000, 3000])
def test_net_moments_match_their_definition(device_lib, n_half):
    xe, xi = _cloud(n_half, 7 + n_half)
    cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
    with api.TreeForce(len(xe), len(xi), cfg) as tf:
        tf.set_tuning(8, 4, 4)
        tf.force(xe, xi)
        d = tf.net_dump()
    xs, cnt, first = d["sorted"], d["count"], d["first"]
    # the sorted particles are the input particles, species kept
    assert np.array_equal(np.sort(xs[:, :3], axis=0), np.sort(np.vstack([xe, xi]), axis=0))
    assert xs[:, 3].sum() == len(xi)
    twig = cnt > 1
    assert cnt[0] == len(xs) and np.all(cnt[~twig] == 1)
    rng = np.random.default_rng(1)
    big = np.flatnonzero(cnt > 64)
    small = np.flatnonzero(twig & (cnt <= 64))
    pick = np.concatenate([big, rng.choice(small, min(3000, len(small)), replace=False)])
    assert np.any(cnt > 2048) and np.any((cnt > 64) & (cnt <= 2048))
    worst = 0.0
    for t in pick:
        p = xs[first[t]:first[t] + cnt[t]]
        X, rec, scale, ext = _reference(p)
        np.testing.assert_allclose(d["centre"][t], X, rtol=0, atol=1e-13 * ext)
        m = d["moments"][t]
        assert m[0] == rec[0] and m[1] == rec[1] and m[5] == rec[5], t
        sel = scale > 0
        err = np.abs(m - rec)[sel] / scale[sel]
        worst = max(worst, float(err.max()))
        assert err.max() <= 1e-11, (t, cnt[t], err.max())
    print(f"net moments n={2 * n_half}: {len(pick)} twigs checked "
          f"({len(big)} above 64 particles), worst scaled error {worst:.2e}")


@pytest.mark.parametrize("colocated", [False, True])
def test_combined_tree_structure(device_lib, colocated):
    """The combined tree's nodes, one thread per node: the root holds every
    particle; each node lies one level below its parent, which precedes it in
    pre-order; a twig's first child follows it; the children of a twig
    partition its particle range in index order; the leaves are the sorted
    particles, one each; and a twig's particles fit the cell of its level
    (the root box halved per level).  colocated: electrons exactly on their
    ions, whose pairs share all 42 spatial levels (chains of one-child
    twigs down to the species bit)."""
    xe, xi = _cloud(20000, 99)
    if colocated:
        xe = xi.copy()
    cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
    with api.TreeForce(len(xe), len(xi), cfg) as tf:
        tf.force(xe, xi)
        d = tf.net_dump()
    n = len(xe) + len(xi)
    first, cnt, lev, par = d["first"], d["count"], d["level"], d["parent"]
    m = len(cnt)
    assert par[0] == -1 and lev[0] == 0 and first[0] == 0 and cnt[0] == n
    i = np.arange(1, m)
    assert np.all((par[1:] >= 0) & (par[1:] < i))
    assert np.all(lev[1:] == lev[par[1:]] + 1)
    leaf = cnt == 1
    twig = ~leaf
    assert leaf.sum() == n
    assert np.array_equal(np.sort(first[leaf]), np.arange(n))
    tw = np.flatnonzero(twig)
    assert np.all(par[tw + 1] == tw)  # pre-order: the first child follows
    # children partition the parent's range, in index order
    ch = np.flatnonzero(par >= 0)
    order = np.lexsort((first[ch], par[ch]))
    ch = ch[order]
    p = par[ch]
    start = np.r_[True, p[1:] != p[:-1]]
    assert np.all(first[ch[start]] == first[p[start]])
    nxt = ~start
    assert np.all(first[ch[nxt]] == first[ch[np.flatnonzero(nxt) - 1]] + cnt[ch[np.flatnonzero(nxt) - 1]])
    sums = np.bincount(p, weights=cnt[ch], minlength=m)
    assert np.array_equal(sums[tw], cnt[tw].astype(float))
    # particles of a twig fit its cell (per axis: root side / 2^level)
    xs = d["sorted"][:, :3]
    side = xs.max(0) - xs.min(0)
    for t in np.random.default_rng(5).choice(tw, min(4000, len(tw)), replace=False):
        q = xs[first[t]:first[t] + cnt[t]]
        ext = q.max(0) - q.min(0)
        assert np.all(ext <= side * 2.0 ** -int(lev[t]) * (1 + 1e-12)), (t, lev[t])
    if colocated:
        assert lev.max() >= 42  # e-i pairs separated only by the species bit
