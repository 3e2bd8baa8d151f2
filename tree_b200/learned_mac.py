"""Trains the learned multipole acceptance criterion on the GPU.

    python -m tree_b200.learned_mac [--n 262144] [--order 3] [--out tree_b200/data/mac_model.npz]

Training data is generated by the method itself: seeded clouds of N = 262,144
particles at electron temperatures across [10, 200] K are evolved a few steps
with the fixed-theta mixed walk, and at each state `tree_gpu_mac_collect`
walks the combined tree with opening angles drawn from [0.2, 0.9], recording
for every tested cell in the acceptance band its features and the exact FP64
error of accepting it.  The network (16 -> 64 -> 64 -> 1) is then trained by
the library's own BF16 tensor-core kernels (`tree_gpu_mac_train`) with a
0.99-quantile pinball loss: the walk uses the prediction to accept cells the
fixed-theta test would open, so an under-estimate is the costly mistake.  The model file holds the FP32 parameters, the feature statistics and
a short training report.
"""
import argparse
import json
import os
import time

import numpy as np

from . import api, cloud, units

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "data", "mac_model.npz")


def model_path(order=3):
    """The shipped model for a far-field order (its labels are the errors of
    that order's expansion)."""
    return DEFAULT_MODEL if order == 3 else os.path.join(HERE, "data", f"mac_model_o{order}.npz")


def collect_and_train(n=262144, te_list=(10.0, 25.0, 50.0, 100.0, 200.0),
                      steps_list=(2, 6, 20), theta=(0.2, 0.9), rho=(0.2, 0.9),
                      max_count=16384, keep=0.1, cap=12_000_000, epochs=10,
                      batch=8192, lr=2e-3, tau=0.99, seed=11, order=3, verbose=True):
    dt = units.dt_code(1e-11)
    half = n // 2
    report = {"n": n, "order": order, "te_list": list(te_list), "steps_list": list(steps_list),
              "theta": list(theta), "rho": list(rho), "max_count": max_count,
              "keep": keep,
              "tau": tau, "epochs": epochs, "batch": batch, "lr": lr, "collects": []}
    t0 = time.time()
    cfg = api.Config(theta=0.5, te=te_list[0], physics=api.PHYS_KELBG,
                     precision=api.PREC_MIXED, mac=api.MAC_FIXED)
    with api.TreeForce(half, half, cfg) as tf:
        tf.set_tuning(8, 4, order)  # labels at the walk's expansion order
        k = 0
        for te in te_list:
            tf.set_config(api.Config(theta=0.5, te=te, physics=api.PHYS_KELBG,
                                     precision=api.PREC_MIXED, mac=api.MAC_FIXED))
            c = cloud.make_cloud(n, seed=seed + int(te), te_k=te)
            tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
            done = 0
            for s in steps_list:
                tf.step(dt, s - done)
                done = s
                k += 1
                tot = tf.mac_collect(theta[0], theta[1], rho[0], rho[1], max_count,
                                     keep, seed * 1000 + k, cap)
                report["collects"].append({"te": te, "step": s, "total": tot})
                if verbose:
                    print(f"collect te={te:g} step={s}: {tot} samples", flush=True)
        t1 = time.time()
        losses = tf.mac_train(epochs, batch, lr, tau, seed)
        t2 = time.time()
        params, stats = tf.mac_get_model()
        feats, labels, extra = tf.mac_samples()
    coef = stats[66:71].astype(np.float64)
    est = (coef[0] * feats[:, 14] + coef[1] * feats[:, 3] + coef[2] * feats[:, 7] +
           coef[3] * feats[:, 6] + coef[4])
    report.update({"samples": int(len(labels)), "collect_s": t1 - t0,
                   "margins": [float(stats[64]), float(stats[65])],
                   "prefilter_coef": [float(c) for c in coef],
                   "corr_label_estimate": float(np.corrcoef(labels, est)[0, 1]),
                   "train_s": t2 - t1, "loss_per_epoch": [float(x) for x in losses],
                   "label_quantiles": {str(q): float(np.quantile(labels, q))
                                       for q in (0.01, 0.1, 0.5, 0.9, 0.99)}})
    if verbose:
        print(json.dumps({k: v for k, v in report.items() if k != "collects"}), flush=True)
    return params, stats, report, (feats, labels, extra)


def save_model(path, params, stats, report):
    """npz with the parameters, statistics and training report, and beside it
    the raw .bin (parameters then statistics, float32) the C++ driver reads."""
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32),
             stats=np.asarray(stats, np.float32),
             report=np.frombuffer(json.dumps(report).encode(), np.uint8))
    write_bin(os.path.splitext(path)[0] + ".bin", params, stats)


def write_bin(path, params, stats):
    np.concatenate([np.asarray(params, "<f4"), np.asarray(stats, "<f4")]).tofile(path)


def load_model(path=DEFAULT_MODEL, order=None):
    """(params, stats, report) of a model file; with `order`, the shipped model
    of that far-field order."""
    if order is not None:
        path = model_path(order)
    d = np.load(path)
    report = json.loads(bytes(d["report"]).decode()) if "report" in d else {}
    return d["params"], d["stats"], report


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--keep", type=float, default=0.1,
                    help="sampling probability of a tested cell in the acceptance band")
    ap.add_argument("--order", type=int, default=3, choices=(2, 3, 4),
                    help="far-field expansion order the labels are computed at")
    ap.add_argument("--out", default="")
    ap.add_argument("--dump-samples", default="")
    args = ap.parse_args()
    out = args.out or model_path(args.order)
    params, stats, report, (f, y, e) = collect_and_train(n=args.n, epochs=args.epochs,
                                                         keep=args.keep, order=args.order)
    save_model(out, params, stats, report)
    if args.dump_samples:
        idx = np.random.default_rng(0).choice(len(y), min(len(y), 150_000), replace=False)
        np.savez_compressed(args.dump_samples, feats=f[idx], labels=y[idx], extra=e[idx])
    print("saved", out)


if __name__ == "__main__":
    main()
