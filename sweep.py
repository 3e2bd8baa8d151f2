"""Long-run measurements of the force path on one GPU.

    python sweep.py precision [--n 1048576] [--steps 1000]
    python sweep.py drift [--n 1048576] [--steps 1000]
    python sweep.py learned [--n 4194304] [--steps 500]

precision: the precision form -- seeded clouds at T_e in {10, 50, 200} K,
    each run with the mixed-precision walk (fixed test, far-field order
    --order, default 3) at opening angles {0.3, 0.5, 0.7} for `steps` steps; at steps 1, 10, 100 and the last, the rms and max
    relative force error against the FP64 O(N^2) direct sum on 16,384 seeded
    targets, and the time per step.
drift: the total energy 1/2 (mv2_el + mv2_ion) + Epot_e + Epot_i, sampled every
    10 steps over `steps` steps from the same seeded cloud, for the
    mixed-precision walk with the learned criterion (--order, --theta, --eta;
    default 3, 0.30, 3e-5) and
    for the plain FP64 fixed-theta path (theta 0.5), or only those named by
    --arms; reports the largest excursion |E - E_0| relative to the mean
    kinetic energy for each.
learned: the learned-MAC form -- the mixed walk with the learned criterion
    (--order, --theta, --eta) for `steps` steps from a seeded cloud at T_e = 50 K;
    at steps 1, 10, 100 and the last, the rms and max relative force error on
    16,384 seeded targets; the time per step, against a fixed-theta mixed walk
    (same theta and order) and the plain FP64 fixed-theta path (theta 0.5) timed over a
    few steps from the final state (after one untimed step each), beside the
    learned walk timed over the same steps from the same state.

One JSON line per run.  Inputs are seeded synthetic clouds (Gaussian at peak
density 1e15 m^-3, electrons on their ions at t = 0, T_i = 1 mK, dt = 1e-11 s).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from tree_b200 import api, cloud, learned_mac, units  # noqa: E402


def _audit(tf, idx):
    st = tf.get_state()
    fd, _ = tf.direct(idx)
    f = np.vstack([st["f_el"], st["f_ion"]])[idx]
    err = np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
    return float(np.sqrt(np.mean(err ** 2))), float(err.max())


def precision(n, steps, seed, tes=(10.0, 50.0, 200.0), thetas=(0.3, 0.5, 0.7), order=3):
    dt = units.dt_code(1e-11)
    rng = np.random.default_rng(seed + 17)
    idx = np.sort(rng.choice(n, min(16384, n), replace=False))
    marks = sorted({m for m in (1, 10, 100, steps) if m <= steps})
    for te in tes:
        c = cloud.make_cloud(n, seed=seed, te_k=te)
        for th in thetas:
            cfg = api.Config(theta=th, te=te, physics=api.PHYS_KELBG, precision=api.PREC_MIXED)
            with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
                tf.set_tuning(8, 4, order)
                tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
                done, rows = 0, []
                t0 = tf.timings()
                wall = 0.0
                for m in marks:
                    w0 = time.perf_counter()
                    tf.step(dt, m - done)
                    wall += time.perf_counter() - w0
                    done = m
                    rms, mx = _audit(tf, idx)
                    rows.append({"step": m, "rms": rms, "max": mx})
                t1 = tf.timings()
            print(json.dumps({"mode": "precision", "n": n, "order": order, "te_k": te, "theta": th,
                              "steps": steps, "audits": rows,
                              "ms_per_step": (t1.ms_total - t0.ms_total) / steps}), flush=True)


def drift(n, steps, seed, nsamp=10, order=3, theta=0.30, eta=3e-5,
          arms_wanted=("mixed_learned", "fp64_plain")):
    dt = units.dt_code(1e-11)
    c = cloud.make_cloud(n, seed=seed)
    params, stats, _ = learned_mac.load_model(order=order)
    out = {"order": order, "theta": theta, "eta": eta}
    arms = (("mixed_learned", api.Config(theta=theta, physics=api.PHYS_KELBG,
                                         precision=api.PREC_MIXED, mac=api.MAC_LEARNED)),
            ("fp64_plain", api.Config(theta=0.5, physics=api.PHYS_KELBG,
                                      precision=api.PREC_FP64)))
    for name, cfg in arms:
        if name not in arms_wanted:
            continue
        with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
            if cfg.precision == api.PREC_MIXED:
                tf.set_tuning(8, 4, order)
                tf.mac_set_model(params, stats)
                tf.mac_config(eta, 0.05, 0.9)
            tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
            t0 = tf.timings()
            rec = tf.run(dt, steps, nsamp=nsamp)
            t1 = tf.timings()
        e = 0.5 * (rec["mv2_el"] + rec["mv2_ion"]) + rec["epot_e"] + rec["epot_i"]
        ke = 0.5 * (rec["mv2_el"] + rec["mv2_ion"])
        out[name] = {"excursion_over_mean_ke": float(np.max(np.abs(e - e[0])) / np.mean(ke)),
                     "e_first": float(e[0]), "e_last": float(e[-1]),
                     "ms_per_step": (t1.ms_total - t0.ms_total) / steps}
    if "mixed_learned" in out and "fp64_plain" in out:
        out["ratio"] = (out["mixed_learned"]["excursion_over_mean_ke"] /
                        out["fp64_plain"]["excursion_over_mean_ke"])
    print(json.dumps({"mode": "drift", "n": n, "steps": steps, "nsamp": nsamp, **out}),
          flush=True)


def learned(n, steps, seed, nplain=3, order=3, theta=0.30, eta=3e-5):
    dt = units.dt_code(1e-11)
    c = cloud.make_cloud(n, seed=seed)
    rng = np.random.default_rng(seed + 17)
    idx = np.sort(rng.choice(n, min(16384, n), replace=False))
    params, stats, _ = learned_mac.load_model(order=order)
    marks = sorted({m for m in (1, 10, 100, steps) if m <= steps})
    cfg = api.Config(theta=theta, physics=api.PHYS_KELBG, precision=api.PREC_MIXED,
                     mac=api.MAC_LEARNED)
    out = {"mode": "learned", "n": n, "steps": steps, "order": order}
    with api.TreeForce(len(c.x_el), len(c.x_ion), cfg) as tf:
        tf.set_tuning(8, 4, order)
        tf.mac_set_model(params, stats)
        tf.mac_config(eta, 0.05, 0.9)
        tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
        done, rows, ms = 0, [], 0.0
        for m in marks:
            t0 = tf.timings()
            tf.step(dt, m - done)
            t1 = tf.timings()
            ms += t1.ms_total - t0.ms_total
            done = m
            rms, mx = _audit(tf, idx)
            rows.append({"step": m, "rms": rms, "max": mx, "n_m2p": t1.n_m2p,
                         "n_p2p": t1.n_p2p, "n_net": t1.n_mac_net})
        st = tf.get_state()
        # the same few steps as the comparison arms, from the same state
        t0 = tf.timings()
        tf.step(dt, nplain)
        t1 = tf.timings()
        out["learned"] = {"theta": theta, "eta": eta, "audits": rows,
                          "ms_per_step": ms / steps,
                          "ms_per_step_from_final_state": (t1.ms_total - t0.ms_total) / nplain}
    # comparison arms from the final state: a few steps each, then an audit
    arms = (("mixed_fixed_same_theta", api.Config(theta=theta, physics=api.PHYS_KELBG,
                                                   precision=api.PREC_MIXED)),
            ("fp64_plain_theta0.5", api.Config(theta=0.5, physics=api.PHYS_KELBG,
                                               precision=api.PREC_FP64)))
    for name, acfg in arms:
        with api.TreeForce(len(c.x_el), len(c.x_ion), acfg) as tf:
            if acfg.precision == api.PREC_MIXED:
                tf.set_tuning(8, 4, order)
            tf.load_state(st["x_el"], st["v_el"], st["f_el"], st["x_ion"], st["v_ion"], st["f_ion"])
            tf.step(dt, 1)  # graph capture and node-array growth, untimed
            t0 = tf.timings()
            tf.step(dt, nplain)
            t1 = tf.timings()
            rms, mx = _audit(tf, idx)
            out[name] = {"ms_per_step": (t1.ms_total - t0.ms_total) / nplain,
                         "steps": nplain, "rms": rms, "max": mx}
    lf = out["learned"]["ms_per_step_from_final_state"]
    out["learned_over_fp64_plain"] = out["fp64_plain_theta0.5"]["ms_per_step"] / lf
    out["learned_over_fixed"] = out["mixed_fixed_same_theta"]["ms_per_step"] / lf
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("mode", choices=["precision", "drift", "learned"])
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--order", type=int, default=3,
                    help="far-field order (precision, drift, learned)")
    ap.add_argument("--arms", default="mixed_learned,fp64_plain",
                    help="drift: the arms to run (the plain FP64 arm does not depend "
                         "on the mixed path's settings)")
    ap.add_argument("--theta", type=float, default=0.30, help="opening angle (drift, learned)")
    ap.add_argument("--eta", type=float, default=3e-5, help="learned budget (drift, learned)")
    args = ap.parse_args()
    if args.mode == "precision":
        precision(args.n or 1048576, args.steps or 1000, args.seed, order=args.order)
    elif args.mode == "drift":
        drift(args.n or 1048576, args.steps or 1000, args.seed, order=args.order,
              theta=args.theta, eta=args.eta, arms_wanted=tuple(args.arms.split(",")))
    else:
        learned(args.n or 4194304, args.steps or 500, args.seed, order=args.order,
                theta=args.theta, eta=args.eta)


if __name__ == "__main__":
    main()
