"""Ensembles of independent clouds in one handle (GPU).

One build (a forest with one root box per cloud), one persistent walk launch
and one integrator launch per step serve every cloud.  Each cloud must come
out exactly as if it had run alone: same tree (its own root box; 39-41
levels below the cloud id instead of 42, which only chains of single-child
cells below co-located e-i pairs reach), same target groups, same
interaction lists, so the same forces bit for bit.
"""
import numpy as np
import pytest

from tree_b200 import api, cloud, learned_mac, units

pytestmark = pytest.mark.gpu

DT = units.dt_code(1e-11)


def _clouds():
    sizes = (3000, 8192, 20002, 50000)
    tes = (10.0, 50.0, 120.0, 200.0)
    n0s = (1e14, 1e15, 3e15, 1e16)
    return [cloud.make_cloud(n, seed=40 + k, te_k=t, n0_per_m3=d)
            for k, (n, t, d) in enumerate(zip(sizes, tes, n0s))], tes


def _cfg(te, theta=0.4, mac=api.MAC_FIXED):
    return api.Config(theta=theta, te=te, physics=api.PHYS_KELBG,
                      precision=api.PREC_MIXED, mac=mac)


def _alone(c, te, nsteps, theta=0.4, mac=api.MAC_FIXED, model=None):
    with api.TreeForce(len(c.x_el), len(c.x_ion), _cfg(te, theta, mac)) as tf:
        if model is not None:
            tf.mac_set_model(*model)
            tf.mac_config(3e-5, 0.05, 0.9)
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        d = tf.step(DT, nsteps) if nsteps else None
        st = tf.get_state()
    x = np.vstack([st["x_el"], st["x_ion"]])
    v = np.vstack([st["v_el"], st["v_ion"]])
    f = np.vstack([st["f_el"], st["f_ion"]])
    return x, v, f, d


@pytest.mark.parametrize("learned", [False, True])
def test_ensemble_equals_clouds_run_alone(device_lib, learned):
    clouds, tes = _clouds()
    x, v, n_el, n_ion = cloud.pack_ensemble(clouds)
    mac = api.MAC_LEARNED if learned else api.MAC_FIXED
    model = None
    if learned:
        params, stats, _ = learned_mac.load_model()
        model = (params, stats)
    with api.Ensemble([_cfg(t, mac=mac) for t in tes], n_el, n_ion) as ens:
        if model is not None:
            ens.mac_set_model(*model)
            ens.mac_config(3e-5, 0.05, 0.9)
        ens.set_state(x, v)
        f0 = ens.get_state()["f"]
        ens.step(DT, 4)
        st = ens.get_state()
        sums = ens.sums()
        if learned:
            assert ens.timings().n_mac_net > 0
    for k, c in enumerate(clouds):
        a, b = ens.offsets[k], ens.offsets[k + 1]
        _, _, fa0, _ = _alone(c, tes[k], 0, mac=mac, model=model)
        np.testing.assert_array_equal(f0[a:b], fa0, err_msg=f"initial force, cloud {k}")
        xa, va, fa, d = _alone(c, tes[k], 4, mac=mac, model=model)
        np.testing.assert_array_equal(st["x"][a:b], xa, err_msg=f"x, cloud {k}")
        np.testing.assert_array_equal(st["v"][a:b], va, err_msg=f"v, cloud {k}")
        np.testing.assert_array_equal(st["f"][a:b], fa, err_msg=f"f, cloud {k}")
        assert sums[k, 0] == pytest.approx(d.epot_e, rel=1e-12, abs=1e-12)
        assert sums[k, 1] == pytest.approx(d.epot_i, rel=1e-12, abs=1e-12)
        assert sums[k, 2] == pytest.approx(d.mv2_el, rel=1e-12)
        assert sums[k, 3] == pytest.approx(d.mv2_ion, rel=1e-12)


def test_ensemble_tiny_ragged_and_empty_clouds(device_lib):
    """Clouds of 2 and 31 particles (one target group each), 33 (a chunked
    root), one species only, and an empty cloud: every non-empty cloud still
    matches its own run alone bit for bit; the empty one contributes nothing."""
    sizes = [(1, 1), (16, 15), (17, 16), (300, 0), (0, 300), (0, 0), (200, 180)]
    rng = np.random.default_rng(77)
    xs, vs = [], []
    for ne, ni in sizes:
        xs.append(rng.standard_normal((ne + ni, 3)) * 20.0)
        vs.append(rng.standard_normal((ne + ni, 3)) * 1e-3)
    n_el = np.array([ne for ne, _ in sizes], np.int64)
    n_ion = np.array([ni for _, ni in sizes], np.int64)
    x, v = np.vstack(xs), np.vstack(vs)
    tes = [20.0 + 10 * k for k in range(len(sizes))]
    with api.Ensemble([_cfg(t) for t in tes], n_el, n_ion) as ens:
        ens.set_state(x, v)
        ens.step(DT, 2)
        st = ens.get_state()
        sums = ens.sums()
    for k, (ne, ni) in enumerate(sizes):
        a, b = ens.offsets[k], ens.offsets[k + 1]
        assert b - a == ne + ni
        if ne + ni == 0:
            assert np.all(sums[k] == 0)
            continue
        with api.TreeForce(ne, ni, _cfg(tes[k])) as tf:
            tf.set_state(xs[k][:ne], vs[k][:ne], xs[k][ne:], vs[k][ne:])
            tf.step(DT, 2)
            sa = tf.get_state()
        np.testing.assert_array_equal(st["x"][a:b], np.vstack([sa["x_el"], sa["x_ion"]]),
                                      err_msg=f"x, cloud {k}")
        np.testing.assert_array_equal(st["f"][a:b], np.vstack([sa["f_el"], sa["f_ion"]]),
                                      err_msg=f"f, cloud {k}")


def test_ensemble_accuracy_per_cloud(device_lib):
    """Every cloud meets the accuracy of the mixed path against its own FP64
    direct sum (cloud-local audit)."""
    clouds, tes = _clouds()
    x, v, n_el, n_ion = cloud.pack_ensemble(clouds)
    with api.Ensemble([_cfg(t, theta=0.3) for t in tes], n_el, n_ion) as ens:
        ens.set_state(x, v)
        ens.step(DT, 3)
        f = ens.get_state()["f"]
        for k in range(len(clouds)):
            a, b = ens.offsets[k], ens.offsets[k + 1]
            rng = np.random.default_rng(k)
            t = np.sort(rng.choice(b - a, min(2048, b - a), replace=False))
            fd, _ = ens.direct(k, t)
            err = np.linalg.norm(f[a:b][t] - fd, axis=1) / np.linalg.norm(fd, axis=1)
            assert np.sqrt(np.mean(err ** 2)) < 1e-4, k


def test_ensemble_rejects_species_split_calls(device_lib):
    clouds, tes = _clouds()
    x, v, n_el, n_ion = cloud.pack_ensemble(clouds[:2])
    with api.Ensemble([_cfg(t) for t in tes[:2]], n_el, n_ion) as ens:
        with pytest.raises(api.TreeGpuError) as ei:
            ens.force(np.zeros((ens.n_el, 3)), np.zeros((ens.n_ion, 3)))
        assert api.ERR[ei.value.code] == "ARG"
        ens.set_state(x, v)
        with pytest.raises(api.TreeGpuError):
            ens.run(DT, 1, rdf=True)
        rec = ens.run(DT, 4, nsamp=2)
        assert list(rec["nloop"]) == [2, 4]
