"""The learned multipole acceptance criterion in the mixed walk (GPU).

The network (16 -> 64 -> 64 -> 1, BF16 tensor cores) predicts the error of
accepting a cell that the fixed opening-angle test would open; the walk
accepts it when the prediction fits the per-target error budget.  These tests
show what that gains over the fixed test (fewer interactions at the same
accuracy against the FP64 direct sum), that it reduces exactly to the fixed
test when it has no model or no budget, and that the on-GPU training loop
runs end to end.
"""
import numpy as np
import pytest

from tree_b200 import api, cloud, learned_mac, units

pytestmark = pytest.mark.gpu

DT = units.dt_code(1e-11)
FLOPS_M2P, FLOPS_P2P = 100, 24  # trace-free octupole M2P, FP32 erf-Kelbg pair


def _evolved_state(n, seed, steps=3):
    """A cloud a few steps after t = 0 (electrons have left their ions)."""
    c = cloud.make_cloud(n, seed=seed)
    cfg = api.Config(theta=0.35, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
    with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        tf.step(DT, steps)
        return tf.get_state()


def _one_step(st, theta, mac, eta=1e-5, model=True, audit=None):
    """One Verlet step from `st`; returns (forces, timings, rms error)."""
    n_el, n_ion = len(st["x_el"]), len(st["x_ion"])
    cfg = api.Config(theta=theta, physics=api.PHYS_KELBG, precision=api.PREC_MIXED,
                     mac=mac)
    with api.TreeForce(n_el, n_ion, cfg) as tf:
        tf.set_tuning(8, 4, 3)
        if mac == api.MAC_LEARNED and model:
            params, stats, _ = learned_mac.load_model()
            tf.mac_set_model(params, stats)
            tf.mac_config(eta, 0.05, 0.9)
        tf.load_state(st["x_el"], st["v_el"], st["f_el"], st["x_ion"], st["v_ion"],
                      st["f_ion"])
        tf.step(DT, 1)
        out = tf.get_state()
        t = tf.timings()
        rms = None
        if audit is not None:
            fd, _ = tf.direct(audit)
            f = np.vstack([out["f_el"], out["f_ion"]])[audit]
            e = np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
            rms = float(np.sqrt(np.mean(e**2)))
    return np.vstack([out["f_el"], out["f_ion"]]), t, rms


def _flops(t):
    return t.n_m2p * FLOPS_M2P + t.n_p2p * FLOPS_P2P


def test_learned_mac_gains_over_fixed_theta(device_lib):
    """At the accuracy the learned criterion reaches, the fixed test needs
    more interactions: the fixed-theta cost curve, interpolated in log-log at
    the learned run's rms error, lies above the learned run's cost."""
    n = 262144
    st = _evolved_state(n, 2024)
    audit = np.sort(np.random.default_rng(5).choice(n, 8192, replace=False))
    _, tl, rms_l = _one_step(st, 0.32, api.MAC_LEARNED, eta=1e-5, audit=audit)
    assert tl.n_mac_net > 0, "the network was never consulted"
    assert rms_l < 1e-4
    curve = []
    for th in (0.26, 0.29, 0.32, 0.35, 0.38, 0.42):
        _, tf_, rms_f = _one_step(st, th, api.MAC_FIXED, audit=audit)
        curve.append((rms_f, _flops(tf_)))
    curve.sort()
    r = np.log([c[0] for c in curve])
    c = np.log([c[1] for c in curve])
    assert r[0] < np.log(rms_l) < r[-1], f"learned rms {rms_l:.3e} outside {curve}"
    fixed_cost = float(np.exp(np.interp(np.log(rms_l), r, c)))
    gain = fixed_cost / _flops(tl)
    assert gain > 1.05, (f"learned: rms {rms_l:.3e} flops {_flops(tl):.3e}; fixed curve "
                         f"{curve}; gain {gain:.3f}")


def test_learned_without_model_is_the_fixed_test(device_lib):
    st = _evolved_state(32768, 9)
    f_fix, t_fix, _ = _one_step(st, 0.4, api.MAC_FIXED)
    f_l, t_l, _ = _one_step(st, 0.4, api.MAC_LEARNED, model=False)
    assert t_l.n_mac_net == 0
    assert (t_l.n_m2p, t_l.n_p2p) == (t_fix.n_m2p, t_fix.n_p2p)
    np.testing.assert_array_equal(f_l, f_fix)


def test_learned_with_no_budget_accepts_nothing_more(device_lib):
    """eta -> 0 leaves no error budget: every decision is the fixed test's,
    so the interaction counts are identical and the forces agree to FP32
    summation-order differences."""
    st = _evolved_state(32768, 10)
    f_fix, t_fix, _ = _one_step(st, 0.4, api.MAC_FIXED)
    f_l, t_l, _ = _one_step(st, 0.4, api.MAC_LEARNED, eta=1e-30)
    assert (t_l.n_m2p, t_l.n_p2p) == (t_fix.n_m2p, t_fix.n_p2p)
    rel = np.linalg.norm(f_l - f_fix, axis=1) / np.linalg.norm(f_fix, axis=1)
    assert rel.max() < 1e-5


def test_learned_budget_orders_accuracy(device_lib):
    """A larger budget accepts more cells and costs accuracy, monotonically."""
    n = 65536
    st = _evolved_state(n, 12)
    audit = np.sort(np.random.default_rng(6).choice(n, 4096, replace=False))
    runs = [_one_step(st, 0.32, api.MAC_LEARNED, eta=eta, audit=audit)
            for eta in (1e-6, 1e-5, 1e-4)]
    flops = [_flops(t) for _, t, _ in runs]
    rms = [r for _, _, r in runs]
    assert flops[0] >= flops[1] >= flops[2]
    assert rms[0] <= rms[1] * 1.05 and rms[1] <= rms[2] * 1.05


def test_collect_and_train_on_gpu(device_lib):
    """Sampling walk -> FP64 labels -> BF16 training, end to end on a small
    cloud; the trained model loads back into a walk."""
    n = 16384
    c = cloud.make_cloud(n, seed=21)
    cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
    with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        tf.step(DT, 3)
        tot = tf.mac_collect(0.2, 0.9, 0.2, 0.9, 16384, 0.5, 7, 400_000)
        feats, labels, extra = tf.mac_samples()
        assert tot >= len(labels) > 1000
        assert np.isfinite(feats).all() and np.isfinite(labels).all()
        theta_g, rho = extra[:, 0], extra[:, 1]
        assert (theta_g >= 0.2).all() and (theta_g <= 0.9).all()
        assert (rho >= 0.2 - 1e-6).all() and (rho <= 0.9 + 1e-6).all()
        # the relative error of a far-field expansion falls with the ratio rho
        lo, hi = labels[rho < 0.35], labels[rho > 0.7]
        assert np.median(lo) < np.median(hi)
        losses = tf.mac_train(3, 4096, 2e-3, 0.9, 3)
        assert np.isfinite(losses).all() and losses[-1] < losses[0]
        params, stats = tf.mac_get_model()
        assert params.shape == (api.MLP_PARAMS,) and np.isfinite(params).all()
        tf.mac_set_model(params, stats)
        tf.mac_config(1e-5, 0.05, 0.9)
        tf.set_config(api.Config(theta=0.32, physics=api.PHYS_KELBG,
                                 precision=api.PREC_MIXED, mac=api.MAC_LEARNED))
        tf.step(DT, 1)
        assert tf.timings().n_mac_net > 0


def test_autotuner_meets_the_accuracy_target(device_lib):
    """The tuner's choice meets the target on the audit and is the fastest
    candidate that does; the handle is left configured with it."""
    from tree_b200.tune import Candidate, autotune
    st = _evolved_state(65536, 14)
    params, stats, _ = learned_mac.load_model()
    space = [Candidate(t, e) for t in (0.3, 0.45, 0.7) for e in (0.0, 3e-5)]
    cfg = api.Config(theta=0.5, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
    with api.TreeForce(len(st["x_el"]), len(st["x_ion"]), cfg) as tf:
        tf.load_state(st["x_el"], st["v_el"], st["f_el"], st["x_ion"], st["v_ion"],
                      st["f_ion"])
        best, trials = autotune(tf, DT, space=space, target=2e-4, audit=4096,
                                model=(params, stats))
        assert len(trials) == len(space)
        assert best is not None and best.rms <= 0.9 * 2e-4
        assert all(t.ms >= best.ms for t in trials if t.rms <= 0.9 * 2e-4)
        assert tf.config.theta == best.cand.theta
        tf.step(DT, 1)
        assert (tf.timings().n_mac_net > 0) == (best.cand.eta > 0)
