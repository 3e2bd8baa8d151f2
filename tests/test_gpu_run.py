"""The step loop on the device: CUDA-graph replay, the reference's sampling
cadence, RDF accumulation and long-run energy conservation (GPU).

main.f90:123-160 runs VVerletNotemp1 -> Force -> VVerletNotemp2 every step,
forms the kinetic sums on steps with Nloop % Nsamp == 0 (vverlet.f90:81-106),
writes TEMPORAL there (sample.f90:55-96) and accumulates the RDF pair counts
of every Force call (tree.f90:918, 1126).  tree_gpu_run does the same with
the state resident on the GPU.
"""
import numpy as np
import pytest

from tree_b200 import api, cloud, learned_mac, units

pytestmark = pytest.mark.gpu

DT = units.dt_code(1e-11)


def _cfg(precision, theta=0.5, mac=api.MAC_FIXED):
    return api.Config(theta=theta, physics=api.PHYS_KELBG, precision=precision, mac=mac)


def _start(n, seed):
    c = cloud.make_cloud(n, seed=seed)
    return c


def _etot(rec):
    return 0.5 * (rec["mv2_el"] + rec["mv2_ion"]) + rec["epot_e"] + rec["epot_i"]


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED])
def test_graph_replay_matches_eager(device_lib, precision):
    """Replaying the captured step body gives the same bits as enqueueing its
    kernels one by one."""
    c = _start(20000, 31)
    out = []
    for graphs in (True, False):
        with api.TreeForce(len(c.x_el), len(c.x_ion), _cfg(precision)) as tf:
            tf.set_graphs(graphs)
            tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
            d = tf.step(DT, 7)
            out.append((tf.get_state(), d.epot_e, d.epot_i, d.mv2_el, tf.timings()))
    (sa, *ea, ta), (sb, *eb, tb) = out
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    assert ea == eb
    assert ta.launches == tb.launches  # the replayed graphs hold the same kernels


def test_run_sampling_cadence_and_values(device_lib):
    """Samples land on Nloop % nsamp == 0 across calls, and each holds the
    same sums a plain step loop ending on that step reports."""
    c = _start(16384, 32)
    cfg = _cfg(api.PREC_FP64)
    with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        r1 = tf.run(DT, 10, nsamp=3)
        r2 = tf.run(DT, 5, nsamp=3)
        assert list(r1["nloop"]) == [3, 6, 9] and list(r2["nloop"]) == [12, 15]
        assert tf.nloop() == 15
    with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        d = tf.step(DT, 9)
    rec = r1[2]
    assert (rec["epot_e"], rec["epot_i"]) == (d.epot_e, d.epot_i)
    assert (rec["mv2_el"], rec["mv2_ion"]) == (d.mv2_el, d.mv2_ion)
    assert (rec["rad_el"], rec["rad_ion"]) == (d.rad_el, d.rad_ion)


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED])
def test_run_rdf_is_the_sum_of_the_force_rdfs(device_lib, precision):
    """RDF counts of a 3-step run equal the sum of the RDF counts of Force at
    the three stepped positions."""
    c = _start(8192, 33)
    cfg = _cfg(precision)
    n_el, n_ion = len(c.x_el), len(c.x_ion)
    with api.TreeForce(n_el, n_ion, cfg) as tf, api.TreeForce(n_el, n_ion, cfg) as tg:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        ref_ei = np.zeros(api.RDF_BINS, np.int64)
        ref_ii = np.zeros(api.RDF_BINS, np.int64)
        st = tf.get_state()
        run_ei = np.zeros(api.RDF_BINS, np.int64)
        run_ii = np.zeros(api.RDF_BINS, np.int64)
        for _ in range(3):
            _, (a, b) = tf.run(DT, 1, rdf=True)
            run_ei += a
            run_ii += b
            st = tf.get_state()
            tg.force(st["x_el"], st["x_ion"], ref_ei, ref_ii)
        np.testing.assert_array_equal(run_ei, ref_ei)
        np.testing.assert_array_equal(run_ii, ref_ii)
        assert run_ei.sum() > 0 and run_ii.sum() > 0


def test_energy_drift_of_mixed_learned_within_twice_the_plain_path(device_lib):
    """1000 steps from the same seeded cloud: the total-energy excursion of
    the mixed-precision walk with the learned MAC stays within 2x that of the
    plain FP64 fixed-theta path (theta = 0.5), for the octupole setting
    (theta 0.30) and the hexadecapole one with local expansions (theta 0.42,
    the N = 1M headline's)."""
    n = 32768
    c = _start(n, 34)
    drift = {}
    arms = (("plain", _cfg(api.PREC_FP64, 0.5), None),
            ("mixed_o3", _cfg(api.PREC_MIXED, 0.30, api.MAC_LEARNED), 3),
            ("mixed_o4", _cfg(api.PREC_MIXED, 0.42, api.MAC_LEARNED), 4))
    for name, cfg, order in arms:
        with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
            if cfg.precision == api.PREC_MIXED:
                params, stats, _ = learned_mac.load_model(order=order)
                tf.set_tuning(8, 4, order)
                tf.mac_set_model(params, stats)
                tf.mac_config(3e-5, 0.05, 0.9)
            tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
            rec = tf.run(DT, 1000, nsamp=10)
        assert len(rec) == 100
        e = _etot(rec)
        scale = np.mean(0.5 * (rec["mv2_el"] + rec["mv2_ion"]))
        drift[name] = float(np.max(np.abs(e - e[0])) / scale)
    assert drift["mixed_o3"] <= 2.0 * drift["plain"] + 1e-6, drift
    assert drift["mixed_o4"] <= 2.0 * drift["plain"] + 1e-6, drift
