"""FP64 device path against the oracle and the golden fixtures (B200).

Parity bar (FP64 mode): tree topology and node values bit-identical to the
oracle's pointer tree; per-particle forces within 1e-10 relative (the device
visits cells in the reference's order, so differences come only from exp /
expm1 / erfc ulps); RDF histograms identical; energies within 1e-12.
"""
import os

import numpy as np
import pytest

import oracle
from tree_b200 import api, cloud, units

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_forces.npz")
FTOL = 1e-10


def _cfg(theta=0.5, physics=api.PHYS_REF, te=50.0, rs=None):
    return api.Config(theta=theta, te=te, rs=rs, physics=physics,
                      precision=api.PREC_FP64, dx_ei=0.01, dx_ii=0.1)


def _oracle_params(cfg):
    lam = units.kelbg_lambdas(cfg.te)
    rs = cfg.rs if cfg.rs is not None else lam[1]
    return oracle.make_params(theta=cfg.theta, rs=rs, dx_ei=cfg.dx_ei,
                              dx_ii=cfg.dx_ii, lambdas=lam,
                              physics=cfg.physics)


def _force_err(f, g):
    """Per-particle |df| / max(|f|, 1e-3 max|f|) (the floor keeps particles
    whose net force cancels to near zero from dominating)."""
    nrm = np.linalg.norm(g, axis=1)
    floor = 1e-3 * max(nrm.max(), 1e-300)
    return np.linalg.norm(f - g, axis=1) / np.maximum(nrm, floor)


def _device_force(x_el, x_ion, cfg):
    with api.TreeForce(len(x_el), len(x_ion), cfg) as tf:
        rei = np.zeros(api.RDF_BINS, np.int64)
        rii = np.zeros(api.RDF_BINS, np.int64)
        f_el, f_ion, ee, ei = tf.force(x_el, x_ion, rei, rii)
        dump = (tf.tree_dump(0), tf.tree_dump(1))
        tm = tf.timings()
    return dict(f_el=f_el, f_ion=f_ion, epot_e=ee, epot_i=ei, rdf_ei=rei,
                rdf_ii=rii, tree=dump, timing=tm)


def _check_tree(dev, ref, theta):
    """Device pre-order dump == oracle pointer-tree dump, bit for bit."""
    assert len(dev["level"]) == len(ref)
    np.testing.assert_array_equal(dev["level"], ref["level"])
    np.testing.assert_array_equal(dev["skip"], ref["skip"])
    leaf = ref["ileaf"] != 0
    np.testing.assert_array_equal(dev["pt"][leaf], ref["pt"][leaf])
    assert np.all(dev["pt"][~leaf] == -1)
    np.testing.assert_array_equal(dev["centre"], ref["xx"])
    mom = np.concatenate([ref["qeff"][:, None], ref["D"], ref["Q"], ref["QQ"]], 1)
    np.testing.assert_array_equal(dev["moments"], mom)
    want_rc = np.where(leaf, -1.0, ref["lx"].max(1) / theta + ref["dx"])
    np.testing.assert_array_equal(dev["rcrit"], want_rc)


@pytest.mark.parametrize("name", ["small_ref", "small_kelbg", "mid_ref", "coloc_ref"])
def test_device_matches_golden(device_lib, name):
    g = np.load(GOLDEN)
    cfg = _cfg(theta=float(g[f"{name}_theta"]), physics=int(g[f"{name}_physics"]),
               te=float(g[f"{name}_te"]), rs=float(g[f"{name}_rs"]))
    d = _device_force(g[f"{name}_x_el"], g[f"{name}_x_ion"], cfg)
    _check_tree(d["tree"][0], g[f"{name}_tree_e"], cfg.theta)
    _check_tree(d["tree"][1], g[f"{name}_tree_i"], cfg.theta)
    f = np.vstack([d["f_el"], d["f_ion"]])
    fr = np.vstack([g[f"{name}_f_el"], g[f"{name}_f_ion"]])
    assert _force_err(f, fr).max() <= FTOL
    np.testing.assert_array_equal(d["rdf_ei"], g[f"{name}_rdf_ei"])
    np.testing.assert_array_equal(d["rdf_ii"], g[f"{name}_rdf_ii"])
    np.testing.assert_allclose([d["epot_e"], d["epot_i"]], g[f"{name}_epot"], rtol=1e-12)


def _displaced(n, seed, shift=0.3):
    c = cloud.make_cloud(n, seed=seed)
    rng = np.random.Generator(np.random.Philox(seed + 7))
    return c.x_ion + rng.standard_normal(c.x_ion.shape) * shift, c.x_ion


@pytest.mark.parametrize("n,seed,theta,physics", [
    (4096, 1, 0.5, api.PHYS_REF),       # config 1 size
    (4096, 2, 0.3, api.PHYS_KELBG),
    (20002, 3, 0.7, api.PHYS_REF),
    (262144, 4, 0.5, api.PHYS_REF),     # config 2 size
])
def test_fp64_forces_match_oracle(device_lib, oracle_lib, n, seed, theta, physics):
    xe, xi = _displaced(n, seed)
    cfg = _cfg(theta=theta, physics=physics)
    d = _device_force(xe, xi, cfg)
    r = oracle.force(xe, xi, _oracle_params(cfg))
    f = np.vstack([d["f_el"], d["f_ion"]])
    fr = np.vstack([r["f_el"], r["f_ion"]])
    err = _force_err(f, fr)
    assert err.max() <= FTOL, f"max rel err {err.max():.3e}"
    np.testing.assert_array_equal(d["rdf_ei"], r["rdf_ei"])
    np.testing.assert_array_equal(d["rdf_ii"], r["rdf_ii"])
    assert d["epot_e"] == pytest.approx(r["epot_e"], rel=1e-12)
    assert d["epot_i"] == pytest.approx(r["epot_i"], rel=1e-12, abs=1e-300)
    assert d["timing"].n_m2p == r["stats"]["n_m2p"]
    assert d["timing"].n_p2p == r["stats"]["n_p2p"]
    if n <= 20002:
        te, _ = oracle.tree_dump(xe, -1)
        _check_tree(d["tree"][0], te, theta)


@pytest.mark.parametrize("n_el,n_ion", [(0, 50), (50, 0), (1, 1), (1, 40), (3, 2), (777, 1234)])
def test_ragged_and_degenerate_species(device_lib, oracle_lib, n_el, n_ion):
    rng = np.random.default_rng(n_el * 1000 + n_ion)
    xe = rng.standard_normal((n_el, 3)) * 20
    xi = rng.standard_normal((n_ion, 3)) * 20
    cfg = _cfg(theta=0.6)
    d = _device_force(xe, xi, cfg)
    r = oracle.force(xe, xi, _oracle_params(cfg))
    f = np.vstack([d["f_el"], d["f_ion"]])
    fr = np.vstack([r["f_el"], r["f_ion"]])
    if len(f):
        assert _force_err(f, fr).max() <= FTOL
    np.testing.assert_array_equal(d["rdf_ei"], r["rdf_ei"])
    if n_el:
        te, _ = oracle.tree_dump(xe, -1)
        _check_tree(d["tree"][0], te, cfg.theta)
    if n_ion:
        ti, _ = oracle.tree_dump(xi, +1)
        _check_tree(d["tree"][1], ti, cfg.theta)


def _stretched_cluster(n_el, n_ion, width, seed):
    """A cluster `width` wide with one particle of each species ~1e3 away: the
    root box is 1e8 cluster widths across, so hundreds of keys share their
    high 64 bits (21 levels) and the build takes its full-key sort."""
    rng = np.random.default_rng(seed)
    xe = rng.standard_normal((n_el, 3)) * width
    xi = rng.standard_normal((n_ion, 3)) * width + 0.3 * width
    xe[0] = (1e3, -2e3, 5e2)
    xi[0] = (-1e3, 1e3, 0.0)
    return xe, xi


def test_tight_cluster_in_a_stretched_box(device_lib, oracle_lib):
    xe, xi = _stretched_cluster(600, 500, 1e-5, 11)
    cfg = _cfg(theta=0.5)
    d = _device_force(xe, xi, cfg)
    r = oracle.force(xe, xi, _oracle_params(cfg))
    f = np.vstack([d["f_el"], d["f_ion"]])
    fr = np.vstack([r["f_el"], r["f_ion"]])
    assert _force_err(f, fr).max() <= FTOL
    np.testing.assert_array_equal(d["rdf_ei"], r["rdf_ei"])
    te, _ = oracle.tree_dump(xe, -1)
    ti, _ = oracle.tree_dump(xi, +1)
    _check_tree(d["tree"][0], te, cfg.theta)
    _check_tree(d["tree"][1], ti, cfg.theta)


def test_rdf_accumulates_across_calls(device_lib):
    xe, xi = _displaced(2000, 9)
    with api.TreeForce(len(xe), len(xi), _cfg()) as tf:
        rei = np.zeros(api.RDF_BINS, np.int64)
        tf.force(xe, xi, rei, None)
        once = rei.copy()
        tf.force(xe, xi, rei, None)
        np.testing.assert_array_equal(rei, 2 * once)


def test_step_matches_oracle_verlet(device_lib, oracle_lib):
    """set_state + step(k) == k x (VVerletNotemp1, Force, VVerletNotemp2)."""
    c = cloud.make_cloud(4096, seed=31)
    cfg = _cfg()
    dt = units.dt_code(1e-11)
    p = _oracle_params(cfg)
    xe, ve, xi, vi = c.x_el.copy(), c.v_el.copy(), c.x_ion.copy(), c.v_ion.copy()
    r = oracle.force(xe, xi, p, rdf=False)
    fe, fi = r["f_el"], r["f_ion"]
    nsteps = 3
    for _ in range(nsteps):
        oracle.kdk1(xe, ve, fe, dt, cfg.xm_el)
        oracle.kdk1(xi, vi, fi, dt, cfg.xm_ion)
        r = oracle.force(xe, xi, p, rdf=False)
        fe, fi = r["f_el"], r["f_ion"]
        oracle.kdk2(ve, fe, dt, cfg.xm_el)
        oracle.kdk2(vi, fi, dt, cfg.xm_ion)
    mv2_e, rad_e = oracle.ke(xe, ve, cfg.xm_el)
    with api.TreeForce(len(xe), len(xi), cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        diag = tf.step(dt, nsteps)
        s = tf.get_state()
    np.testing.assert_allclose(s["x_el"], xe, rtol=0, atol=1e-10 * np.abs(xe).max())
    np.testing.assert_allclose(s["x_ion"], xi, rtol=0, atol=1e-12 * np.abs(xi).max())
    np.testing.assert_allclose(s["v_el"], ve, rtol=0, atol=1e-9 * np.abs(ve).max())
    np.testing.assert_allclose(s["v_ion"], vi, rtol=0, atol=1e-9 * np.abs(vi).max())
    assert diag.mv2_el == pytest.approx(mv2_e, rel=1e-9)
    assert diag.rad_el == pytest.approx(rad_e, rel=1e-9)
    assert diag.epot_e == pytest.approx(r["epot_e"], rel=1e-9)


def test_duplicate_positions_report_depth_error(device_lib):
    x = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [2.0, 0.0, 1.0]])
    xi = np.array([[0.5, 0.5, 0.5], [3.0, 1.0, 0.0]])
    with api.TreeForce(len(x), len(xi), _cfg()) as tf:
        with pytest.raises(api.TreeGpuError) as ei:
            tf.force(x, xi)
        assert ei.value.code == -2
        # the handle stays usable
        x[2] += 1e-3
        f_el, _, _, _ = tf.force(x, xi)
        assert np.all(np.isfinite(f_el))


def test_nonfinite_position_is_rejected(device_lib):
    x = np.array([[0.0, 0.0, 0.0], [np.nan, 1.0, 1.0]])
    xi = np.array([[0.5, 0.5, 0.5], [3.0, 1.0, 0.0]])
    with api.TreeForce(2, 2, _cfg()) as tf:
        with pytest.raises(api.TreeGpuError) as ei:
            tf.force(x, xi)
        assert ei.value.code == -3


@pytest.mark.parametrize("physics", [api.PHYS_REF, api.PHYS_KELBG])
def test_direct_sum_judge_matches_oracle(device_lib, oracle_lib, physics):
    xe, xi = _displaced(20000, 41)
    cfg = _cfg(physics=physics)
    rng = np.random.default_rng(5)
    n_el = len(xe)
    t = np.sort(rng.choice(len(xe) + len(xi), 700, replace=False))
    with api.TreeForce(len(xe), len(xi), cfg) as tf:
        tf.force(xe, xi)
        f, e = tf.direct(t)
    r = oracle.direct(xe, xi, _oracle_params(cfg), t[t < n_el], t[t >= n_el] - n_el)
    fr = np.vstack([r["f_el"], r["f_ion"]])
    assert _force_err(f, fr).max() <= 1e-12
    assert e.sum() == pytest.approx(r["epot"], rel=1e-12)


def test_direct_sum_is_theta_zero_walk(device_lib):
    xe, xi = _displaced(3000, 42)
    cfg = _cfg(theta=1e-12, physics=api.PHYS_KELBG)
    with api.TreeForce(len(xe), len(xi), cfg) as tf:
        f_el, f_ion, ee, ei = tf.force(xe, xi)
        f, e = tf.direct(np.arange(len(xe) + len(xi)))
    fw = np.vstack([f_el, f_ion])
    assert _force_err(fw, f).max() <= 1e-12
    assert ee + ei == pytest.approx(e.sum(), rel=1e-12)
