"""Mixed-precision warp-group walk (B200) against the FP64 judges.

The mixed path is not bit-comparable with the reference (different moments,
group MAC, FP32 arithmetic); its bar is accuracy against the FP64 O(N^2)
direct sum with the same pair laws, checked both with the device judge and
with the CPU oracle's direct sum.
"""
import numpy as np
import pytest

import oracle
from tree_b200 import api, cloud, units

pytestmark = pytest.mark.gpu


def _displaced(n, seed, shift=0.3):
    c = cloud.make_cloud(n, seed=seed)
    rng = np.random.Generator(np.random.Philox(seed + 7))
    return c.x_ion + rng.standard_normal(c.x_ion.shape) * shift, c.x_ion


def _rel(f, g):
    return np.linalg.norm(f - g, axis=1) / np.linalg.norm(g, axis=1)


def _mixed(theta=0.5, physics=api.PHYS_KELBG):
    return api.Config(theta=theta, physics=physics, precision=api.PREC_MIXED)


@pytest.mark.parametrize("physics", [api.PHYS_KELBG, api.PHYS_REF])
def test_mixed_theta_zero_equals_direct_sum(device_lib, physics):
    """With every cell opened the walk is a pure particle sum in FP32 with
    hi/lo offsets and compensated accumulation."""
    xe, xi = _displaced(6000, 3)
    with api.TreeForce(len(xe), len(xi), _mixed(1e-9, physics)) as tf:
        f_el, f_ion, ee, ei = tf.force(xe, xi)
        assert tf.timings().n_m2p == 0
        fd, ed = tf.direct(np.arange(len(xe) + len(xi)))
    f = np.vstack([f_el, f_ion])
    err = _rel(f, fd)
    assert np.sqrt(np.mean(err**2)) < 2e-6 and err.max() < 1e-4
    assert ee + ei == pytest.approx(ed.sum(), rel=1e-5)


@pytest.mark.parametrize("n,theta,rms_bound", [(8192, 0.5, 1e-4), (65536, 0.5, 1e-4),
                                              (65536, 0.7, 5e-4)])
def test_mixed_accuracy_vs_device_direct_sum(device_lib, n, theta, rms_bound):
    xe, xi = _displaced(n, 11)
    rng = np.random.default_rng(1)
    t = np.sort(rng.choice(n, min(n, 4096), replace=False))
    with api.TreeForce(len(xe), len(xi), _mixed(theta)) as tf:
        f_el, f_ion, _, _ = tf.force(xe, xi)
        fd, _ = tf.direct(t)
    f = np.vstack([f_el, f_ion])[t]
    err = _rel(f, fd)
    rms = float(np.sqrt(np.mean(err**2)))
    assert rms < rms_bound, f"rms {rms:.3e}"
    assert err.max() < 100 * rms_bound


def test_mixed_matches_oracle_direct_sum(device_lib, oracle_lib):
    """Independent judge: the CPU oracle's FP64 direct sum."""
    xe, xi = _displaced(4096, 12)
    lam = units.kelbg_lambdas(50.0)
    p = oracle.make_params(theta=1e-12, rs=lam[1], lambdas=lam,
                           physics=oracle.PHYS_KELBG)
    d = oracle.direct(xe, xi, p)
    with api.TreeForce(len(xe), len(xi), _mixed(0.5)) as tf:
        f_el, f_ion, ee, ei = tf.force(xe, xi)
    err = _rel(np.vstack([f_el, f_ion]), np.vstack([d["f_el"], d["f_ion"]]))
    assert np.sqrt(np.mean(err**2)) < 1e-4
    assert ee + ei == pytest.approx(d["epot"], rel=1e-4)


def test_mixed_more_accurate_than_reference_moments(device_lib):
    """Exact quadrupoles + group MAC beat the one-level moments of the FP64
    parity path at the same theta."""
    xe, xi = _displaced(65536, 13, shift=2.0)
    rng = np.random.default_rng(2)
    t = np.sort(rng.choice(65536, 2048, replace=False))
    out = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=prec)
        with api.TreeForce(len(xe), len(xi), cfg) as tf:
            f_el, f_ion, _, _ = tf.force(xe, xi)
            fd, _ = tf.direct(t)
        err = _rel(np.vstack([f_el, f_ion])[t], fd)
        out[prec] = np.sqrt(np.mean(err**2))
    assert out[api.PREC_MIXED] < out[api.PREC_FP64]


@pytest.mark.parametrize("n_el,n_ion", [(0, 70), (70, 0), (1, 1), (1, 33), (33, 1), (31, 65)])
def test_mixed_ragged_species(device_lib, n_el, n_ion):
    rng = np.random.default_rng(n_el * 100 + n_ion)
    xe = rng.standard_normal((n_el, 3)) * 20
    xi = rng.standard_normal((n_ion, 3)) * 20
    with api.TreeForce(n_el, n_ion, _mixed(0.5)) as tf:
        f_el, f_ion, _, _ = tf.force(xe, xi)
        fd, _ = tf.direct(np.arange(n_el + n_ion))
    f = np.vstack([f_el, f_ion])
    assert np.all(np.isfinite(f))
    if n_el + n_ion > 1:
        assert np.sqrt(np.mean(_rel(f, fd) ** 2)) < 1e-4


def test_mixed_tight_cluster_in_a_stretched_box(device_lib):
    """Hundreds of keys share their high 64 bits (a cluster 0.3 um wide in a
    box 3e6 um wide), which takes the build's full-key sort: the forces meet
    the accuracy bar and do not depend on the input order within a species."""
    rng = np.random.default_rng(12)
    xe = rng.standard_normal((300, 3)) * 0.3
    xi = rng.standard_normal((300, 3)) * 0.3
    xe[0] = (1e6, -2e6, 5e5)
    xi[0] = (-1e6, 1e6, 0.0)
    pe = np.concatenate([[0], 1 + rng.permutation(299)])
    pi = np.concatenate([[0], 1 + rng.permutation(299)])
    with api.TreeForce(300, 300, _mixed(0.5)) as tf:
        f_el, f_ion, _, _ = tf.force(xe, xi)
        fd, _ = tf.direct(np.arange(600))
        g_el, g_ion, _, _ = tf.force(xe[pe], xi[pi])
    f = np.vstack([f_el, f_ion])
    assert np.all(np.isfinite(f))
    assert np.sqrt(np.mean(_rel(f, fd) ** 2)) < 1e-4
    np.testing.assert_array_equal(g_el, f_el[pe])
    np.testing.assert_array_equal(g_ion, f_ion[pi])


def test_mixed_step_energy_drift_close_to_fp64(device_lib):
    """50 steps of dt = 1e-11 s: the mixed path's relative energy drift stays
    within a small multiple of the FP64 path's."""
    c = cloud.make_cloud(8192, seed=21)
    dt = units.dt_code(1e-11)
    drift = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=prec)
        with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
            tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
            d0 = tf.step(dt, 5)
            e0 = 0.5 * (d0.mv2_el + d0.mv2_ion) + d0.epot_e + d0.epot_i
            d1 = tf.step(dt, 50)
            e1 = 0.5 * (d1.mv2_el + d1.mv2_ion) + d1.epot_e + d1.epot_i
        drift[prec] = abs(e1 - e0) / abs(0.5 * (d1.mv2_el + d1.mv2_ion))
    assert drift[api.PREC_MIXED] < 2 * drift[api.PREC_FP64] + 1e-6, drift


def test_mixed_rdf_counts_pairs(device_lib):
    xe, xi = _displaced(4096, 14)
    with api.TreeForce(len(xe), len(xi), _mixed(1e-9)) as tf:
        rei = np.zeros(api.RDF_BINS, np.int64)
        rii = np.zeros(api.RDF_BINS, np.int64)
        tf.force(xe, xi, rei, rii)
    # theta -> 0: every e-i pair is a leaf pair, counted once per target side
    d = np.linalg.norm(xe[:, None, :] - xi[None, :, :], axis=2)
    want = 2 * np.bincount(np.minimum((d / 0.01).astype(np.int64), 10001).ravel(),
                           minlength=10002)[:10001]
    # bins come from the FP32 distance (about 1e-6 relative): a pair that
    # close to a bin edge may be counted in the neighbouring bin, so the
    # totals agree and the cumulative counts differ by a few such pairs
    assert abs(int(rei.sum()) - int(want.sum())) <= 1e-4 * want.sum()
    assert np.abs(np.cumsum(rei) - np.cumsum(want)).max() <= 2e-3 * want.sum()
    assert np.abs(rei - want).sum() <= 1e-2 * want.sum()


def test_far_field_orders_converge(device_lib):
    """A neutral cluster (50 electrons, 50 ions in [-1, 1]^3) and one target
    5.5 cluster half-widths away along each axis in turn, so that the target's
    force is the cluster's field alone and the truncation error of the
    accepted cells (about a quarter of the cluster each, extent over distance
    about 0.2) stays far above FP32 rounding: the error falls with each
    expansion order (quadrupole, octupole, hexadecapole)."""
    rng = np.random.default_rng(31)
    src_e = rng.uniform(-1.0, 1.0, (50, 3))
    src_i = rng.uniform(-1.0, 1.0, (50, 3))
    tgts = [np.array(v) for v in ((5.5, 0.1, -0.2), (-5.5, 0.3, 0.1), (0.2, 5.5, 0.1),
                                  (-0.1, -5.5, 0.2), (0.1, -0.2, 5.5), (0.3, 0.1, -5.5))]
    errs = {}
    for order in (2, 3, 4):
        rel = []
        for k, t in enumerate(tgts):
            ion = k % 2 == 1
            xe = src_e if ion else np.vstack([src_e, t[None]])
            xi = np.vstack([src_i, t[None]]) if ion else src_i
            target = len(xe) + 50 if ion else 50
            with api.TreeForce(len(xe), len(xi), _mixed(0.9)) as tf:
                tf.set_tuning(1, 4, order)  # bucket 1: every accepted cell is a multipole
                f_el, f_ion, _, _ = tf.force(xe, xi)
                assert tf.timings().n_m2p > 0
                fd, _ = tf.direct(np.array([target]))
            f = np.vstack([f_el, f_ion])[[target]]
            rel.append(float(_rel(f, fd)[0]))
        errs[order] = float(np.sqrt(np.mean(np.square(rel))))
    assert errs[4] > 1e-6, errs  # truncation, not FP32 rounding
    assert errs[3] < 0.5 * errs[2] and errs[4] < 0.5 * errs[3], errs


@pytest.mark.parametrize("theta", [0.5, 0.7])
def test_hexadecapole_more_accurate_than_octupole(device_lib, theta):
    xe, xi = _displaced(65536, 17, shift=1.0)
    rng = np.random.default_rng(3)
    t = np.sort(rng.choice(65536, 4096, replace=False))
    rms = {}
    for order in (3, 4):
        with api.TreeForce(len(xe), len(xi), _mixed(theta)) as tf:
            tf.set_tuning(8, 4, order)
            f_el, f_ion, _, _ = tf.force(xe, xi)
            fd, _ = tf.direct(t)
        rms[order] = float(np.sqrt(np.mean(_rel(np.vstack([f_el, f_ion])[t], fd) ** 2)))
    assert rms[4] < 0.7 * rms[3], rms


def test_local_expansion_of_far_cells(device_lib):
    """Accepted cells far from a target group are summed into the group's
    local expansion instead of being evaluated per target: a large share of
    the far field moves there while the error against the direct sum, the
    forces and the potential energy stay where they were."""
    n = 262144
    xe, xi = _displaced(n, 21, shift=1.0)
    rng = np.random.default_rng(4)
    t = np.sort(rng.choice(n, 8192, replace=False))
    out = {}
    fd = None
    for eps in (0.0, 0.08):
        with api.TreeForce(len(xe), len(xi), _mixed(0.42)) as tf:
            tf.set_tuning(8, 4, 4)
            tf.set_local_expansion(eps)
            f_el, f_ion, ee, ei = tf.force(xe, xi)
            tm = tf.timings()
            if fd is None:
                fd, _ = tf.direct(t)
        f = np.vstack([f_el, f_ion])
        out[eps] = (f, ee + ei, tm.n_m2p, tm.n_local, np.sqrt(np.mean(_rel(f[t], fd) ** 2)))
    f0, e0, m2p0, loc0, rms0 = out[0.0]
    f1, e1, m2p1, loc1, rms1 = out[0.08]
    assert loc0 == 0 and loc1 > 0
    # per-target far-field evaluations fall by a fifth or more
    assert m2p1 < 0.8 * m2p0
    assert rms1 < 1.1 * rms0 + 2e-6 and rms1 < 1e-4, (rms0, rms1)
    d = _rel(f1, f0)
    assert np.sqrt(np.mean(d**2)) < 3e-5 and d.max() < 2e-3
    assert e1 == pytest.approx(e0, rel=1e-5)
    with api.TreeForce(8, 8, _mixed(0.5)) as tf:
        with pytest.raises(api.TreeGpuError):
            tf.set_local_expansion(0.6)
