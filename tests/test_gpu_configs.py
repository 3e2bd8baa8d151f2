"""The two plain-method workloads run as specified, FP64 device path against
the oracle (B200).

Plain method, N = 4,096: 2,048 electrons on 2,048 ions (88 amu) at t = 0,
Gaussian of sigma = 64 um (peak density 1e15 m^-3), Maxwellian T_e = 50 K,
T_i = 1 mK, theta = 0.5, dt = 1e-11 s, 100 velocity-Verlet steps.  The
reference loop is main.f90:123-131 (VVerletNotemp1 -> Force ->
VVerletNotemp2, vverlet.f90:9-112).

Plain method, N = 262,144: the same construction at sigma = 255 um; forces
compared with the reference algorithm at step 0 and at step 1,000.  The late
state is the one where the device's 42-level keys and the expanded root box
(electrons ejected by dt = 1e-11 s, bounding box grown by orders of
magnitude) could part from the reference's unbounded insertion
(tree.f90:128-273).

The pair laws are the reference's (Coulomb e-e / i-i with the r^2 > 0.01
cutoff, exp-screened e-i with rs = lambda_ei), rs being the one free choice.
"""
import numpy as np
import pytest

import oracle
from tree_b200 import api, cloud, units

pytestmark = pytest.mark.gpu
FTOL = 1e-10


def _cfg(theta=0.5):
    return api.Config(theta=theta, te=50.0, physics=api.PHYS_REF,
                      precision=api.PREC_FP64, dx_ei=0.01, dx_ii=0.1)


def _oracle_params(cfg):
    lam = units.kelbg_lambdas(cfg.te)
    return oracle.make_params(theta=cfg.theta, rs=lam[1], dx_ei=cfg.dx_ei,
                              dx_ii=cfg.dx_ii, lambdas=lam, physics=cfg.physics)


def _force_err(f, g):
    nrm = np.linalg.norm(g, axis=1)
    floor = 1e-3 * max(nrm.max(), 1e-300)
    return np.linalg.norm(f - g, axis=1) / np.maximum(nrm, floor)


def _check_tree(dev, ref, theta):
    assert len(dev["level"]) == len(ref)
    np.testing.assert_array_equal(dev["level"], ref["level"])
    np.testing.assert_array_equal(dev["skip"], ref["skip"])
    leaf = ref["ileaf"] != 0
    np.testing.assert_array_equal(dev["pt"][leaf], ref["pt"][leaf])
    np.testing.assert_array_equal(dev["centre"], ref["xx"])
    mom = np.concatenate([ref["qeff"][:, None], ref["D"], ref["Q"], ref["QQ"]], 1)
    np.testing.assert_array_equal(dev["moments"], mom)
    want_rc = np.where(leaf, -1.0, ref["lx"].max(1) / theta + ref["dx"])
    np.testing.assert_array_equal(dev["rcrit"], want_rc)


def _compare_force(tf, x_el, x_ion, cfg, p, trees=True):
    """Device Force on (x_el, x_ion) against the oracle's on the same positions:
    forces per particle, energies, RDF histograms, interaction counts and
    (optionally) both trees node for node."""
    rei = np.zeros(api.RDF_BINS, np.int64)
    rii = np.zeros(api.RDF_BINS, np.int64)
    f_el, f_ion, ee, ei = tf.force(x_el, x_ion, rei, rii)
    tm = tf.timings()
    r = oracle.force(x_el, x_ion, p)
    f = np.vstack([f_el, f_ion])
    fr = np.vstack([r["f_el"], r["f_ion"]])
    err = _force_err(f, fr)
    assert err.max() <= FTOL, f"max rel force err {err.max():.3e}"
    np.testing.assert_array_equal(rei, r["rdf_ei"])
    np.testing.assert_array_equal(rii, r["rdf_ii"])
    assert ee == pytest.approx(r["epot_e"], rel=1e-12)
    assert ei == pytest.approx(r["epot_i"], rel=1e-12, abs=1e-300)
    assert tm.n_m2p == r["stats"]["n_m2p"]
    assert tm.n_p2p == r["stats"]["n_p2p"]
    if trees:
        te, _ = oracle.tree_dump(x_el, -1)
        ti, _ = oracle.tree_dump(x_ion, +1)
        _check_tree(tf.tree_dump(0), te, cfg.theta)
        _check_tree(tf.tree_dump(1), ti, cfg.theta)
    return float(err.max())


def test_plain_method_4096_every_step_of_100(device_lib, oracle_lib):
    """Each of the 100 device steps (tree_gpu_step) equals one reference step
    taken from the device's own previous state: the drift and both kicks bit
    for bit, the forces within 1e-10, and at the end identical trees, RDF and
    interaction counts."""
    c = cloud.make_cloud(4096, seed=101)
    assert np.array_equal(c.x_el, c.x_ion)  # electrons start on their ions
    cfg = _cfg()
    p = _oracle_params(cfg)
    dt = units.dt_code(1e-11)
    with api.TreeForce(2048, 2048, cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        s = tf.get_state()
        r0 = oracle.force(c.x_el, c.x_ion, p, rdf=False)
        f0 = np.vstack([s["f_el"], s["f_ion"]])
        assert _force_err(f0, np.vstack([r0["f_el"], r0["f_ion"]])).max() <= FTOL
        worst = 0.0
        for k in range(100):
            xe, ve, fe = s["x_el"].copy(), s["v_el"].copy(), s["f_el"].copy()
            xi, vi, fi = s["x_ion"].copy(), s["v_ion"].copy(), s["f_ion"].copy()
            oracle.kdk1(xe, ve, fe, dt, cfg.xm_el)
            oracle.kdk1(xi, vi, fi, dt, cfg.xm_ion)
            tf.step(dt, 1)
            s = tf.get_state()
            np.testing.assert_array_equal(s["x_el"], xe, err_msg=f"step {k + 1}")
            np.testing.assert_array_equal(s["x_ion"], xi, err_msg=f"step {k + 1}")
            r = oracle.force(xe, xi, p, rdf=False)
            f = np.vstack([s["f_el"], s["f_ion"]])
            fr = np.vstack([r["f_el"], r["f_ion"]])
            err = _force_err(f, fr).max()
            worst = max(worst, err)
            assert err <= FTOL, f"step {k + 1}: max rel force err {err:.3e}"
            # the second kick on the device's forces, for the velocities
            oracle.kdk2(ve, s["f_el"], dt, cfg.xm_el)
            oracle.kdk2(vi, s["f_ion"], dt, cfg.xm_ion)
            np.testing.assert_array_equal(s["v_el"], ve, err_msg=f"step {k + 1}")
            np.testing.assert_array_equal(s["v_ion"], vi, err_msg=f"step {k + 1}")
        # the final state once more through Force, with RDF, counts and trees
        _compare_force(tf, s["x_el"], s["x_ion"], cfg, p)
    print(f"plain method N=4096: worst per-step force error over 100 steps {worst:.2e}")


def test_plain_method_4096_free_run_of_100(device_lib, oracle_lib):
    """100 steps in one tree_gpu_step call (CUDA-graph replays) against the
    oracle's own 100-step loop from the same start: positions, velocities and
    the kinetic sums of the last step."""
    c = cloud.make_cloud(4096, seed=101)
    cfg = _cfg()
    p = _oracle_params(cfg)
    dt = units.dt_code(1e-11)
    xe, ve, xi, vi = c.x_el.copy(), c.v_el.copy(), c.x_ion.copy(), c.v_ion.copy()
    r = oracle.force(xe, xi, p, rdf=False)
    fe, fi = r["f_el"], r["f_ion"]
    for _ in range(100):
        oracle.kdk1(xe, ve, fe, dt, cfg.xm_el)
        oracle.kdk1(xi, vi, fi, dt, cfg.xm_ion)
        r = oracle.force(xe, xi, p, rdf=False)
        fe, fi = r["f_el"], r["f_ion"]
        oracle.kdk2(ve, fe, dt, cfg.xm_el)
        oracle.kdk2(vi, fi, dt, cfg.xm_ion)
    mv2_e, rad_e = oracle.ke(xe, ve, cfg.xm_el)
    mv2_i, rad_i = oracle.ke(xi, vi, cfg.xm_ion)
    with api.TreeForce(2048, 2048, cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        diag = tf.step(dt, 100)
        s = tf.get_state()
    dx_e = np.abs(s["x_el"] - xe).max() / np.abs(xe).max()
    dv_e = np.abs(s["v_el"] - ve).max() / np.abs(ve).max()
    print(f"plain method N=4096 free run: max |dx|/max|x| {dx_e:.2e}, "
          f"max |dv|/max|v| {dv_e:.2e}")
    np.testing.assert_allclose(s["x_el"], xe, rtol=0, atol=1e-9 * np.abs(xe).max())
    np.testing.assert_allclose(s["x_ion"], xi, rtol=0, atol=1e-9 * np.abs(xi).max())
    np.testing.assert_allclose(s["v_el"], ve, rtol=0, atol=1e-9 * np.abs(ve).max())
    np.testing.assert_allclose(s["v_ion"], vi, rtol=0, atol=1e-9 * np.abs(vi).max())
    assert diag.mv2_el == pytest.approx(mv2_e, rel=1e-9)
    assert diag.mv2_ion == pytest.approx(mv2_i, rel=1e-9)
    assert diag.rad_el == pytest.approx(rad_e, rel=1e-9)
    assert diag.rad_ion == pytest.approx(rad_i, rel=1e-9)
    assert diag.epot_e == pytest.approx(r["epot_e"], rel=1e-9)


def test_plain_method_262144_steps_0_and_1000(device_lib, oracle_lib):
    """Forces against the oracle on the co-located start (step 0) and on the
    device's state after 1,000 steps, each with identical trees, RDF and
    interaction counts."""
    c = cloud.make_cloud(262144, seed=202)
    assert abs(c.sigma_um - 255.0) < 1.0
    cfg = _cfg()
    p = _oracle_params(cfg)
    dt = units.dt_code(1e-11)
    with api.TreeForce(131072, 131072, cfg) as tf:
        e0 = _compare_force(tf, c.x_el, c.x_ion, cfg, p)
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        tf.step(dt, 1000)
        assert tf.nloop() == 1000
        s = tf.get_state()
        ext = max(np.abs(s["x_el"]).max(), np.abs(s["x_ion"]).max())
        e1000 = _compare_force(tf, s["x_el"], s["x_ion"], cfg, p)
    print(f"plain method N=262144: step 0 max err {e0:.2e}; step 1000 max err {e1000:.2e}, "
          f"largest |x| {ext:.3e} um (sigma {c.sigma_um:.1f} um)")
