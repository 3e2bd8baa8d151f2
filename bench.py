#!/usr/bin/env python
"""Benchmark of the TREE force path: particle-steps/s at N = 1,048,576.

One step = VVerletNotemp1 -> Force (octree build + upward pass + tree walk,
with the e-i / i-i RDF pair counts of every step) -> VVerletNotemp2, the loop
body of main.f90:123-131 of hpjeonGIT/TREE, with the TEMPORAL kinetic sums on
every step with Nloop % nsamp == 0 (vverlet.f90:81-106); the timed loop is
one tree_gpu_run call.  Workload: a seeded synthetic ultracold-plasma cloud
(isotropic Gaussian of ions at peak density 1e15 m^-3 with each electron
starting on its ion, T_e = 50 K, T_i = 1 mK, dt = 1e-11 s, erf-Kelbg pair
laws).  The inputs (positions, velocities, trees) are far larger than the
126 MB L2 and every step rebuilds the trees from scratch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the CPU restatement of the reference algorithm
(pointer octree, serial insertion, recursive OpenMP walks in FP64) on all host
cores, on the same workload configuration (opening angle, pair laws, RDF
every step): whole steps from the t = 0 cloud after the untimed initial force
(Vinit), until K steps or the time budget --ref-budget, whichever comes
first; the line reports the steps it actually timed.
With N > 1 GPUs every rank runs an independent replica of the workload (the
path has no exchange step); value = all particles x steps / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at N=1,048,576 (force path: build + upward + walk + KDK)"
UNIT = "particle-steps/s"
DT_S = 1e-11

# Algorithmic flops per interaction, counted from the kernels' formulas
# (FMA = 2; divisions, square roots and exponentials count as one flop each).
FLOPS_M2P_REF = 194    # tree.f90:736-779 evaluated literally (FP64 path)
FLOPS_P2P_REF = 30     # leaf laws of tree.f90 / erf-Kelbg with the x^2>40 shortcut
FLOPS_M2P_MIXED = {2: 50, 3: 100, 4: 195}  # FP32 trace-free far field to order 2 / 3 / 4
FLOPS_P2P_MIXED = 24   # FP32 erf-Kelbg pair with hi/lo offsets
FLOPS_MLP = 2 * (16 * 64 + 64 * 64 + 64)  # one learned-MAC evaluation (BF16 mma + FP32)
# One far cell summed into a target group's local expansion (local.cuh at
# order 4: potential and its first to fourth derivatives, ~700 operations of
# which most are FMA), evaluated once per group instead of once per target.
FLOPS_LOCAL = 1250
RDF_BYTES = 2 * 10001 * 8  # the two 64-bit RDF histograms read back per call
SAMPLE_BYTES = 48          # one TEMPORAL record

# Headline configuration: mixed precision, learned MAC on top of theta = 0.42,
# hexadecapole far field; chosen so the rms relative force error against the
# FP64 direct sum stays below 1e-4 at this workload with a margin (7.2e-5 at
# the state after 25 steps in the tuning sweep; the accuracy audit below,
# which every run reports, measures it again).
HEADLINE = dict(theta=0.42, eta=3e-5, order=4, bucket=8, loc=0.08)
# Fixed-theta arms beside the learned criterion, per far-field order: the
# opening angles around the one that meets 1e-4 without the learned test.
FIXED_ARMS = {2: (0.20, 0.22, 0.25), 3: (0.30, 0.32, 0.35), 4: (0.40, 0.42, 0.45)}
# Opening angles the ensemble autotuner tries, per far-field order.
TUNE_THETAS = {2: (0.14, 0.16, 0.18, 0.20, 0.22), 3: (0.20, 0.22, 0.24, 0.26, 0.28, 0.30),
               4: (0.30, 0.33, 0.36, 0.39, 0.42, 0.45)}
# Ensemble of 64 clouds, fixed here so that the bench does no tuning: the
# learned criterion on the hexadecapole far field at theta = 0.36, eta = 3e-5
# (worst cloud rms 5.7e-5 on 4,096 targets each, 10 steps after the 13-step
# warm-up; the tuner's fastest order-4 pick, fixed theta = 0.39, reached
# 1.09e-4 on one cloud at that audit), two blocks per SM (the learned build's
# register budget).
ENSEMBLE_TUNED = dict(theta=0.36, eta=3e-5, bucket=8, order=4, blocks_per_sm=2)
# The fixed test's own grid (its 80-register build holds three blocks per SM).
ENSEMBLE_FIXED_BPS = 3


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    # --particles: the same, for launchers (torchrun) that claim --n* options
    ap.add_argument("--n", "--particles", dest="n", type=int, default=1048576)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--mac", choices=["fixed", "learned"], default="learned")
    ap.add_argument("--physics", choices=["kelbg", "ref"], default="kelbg")
    ap.add_argument("--theta", type=float, default=HEADLINE["theta"])
    ap.add_argument("--eta", type=float, default=HEADLINE["eta"])
    ap.add_argument("--order", type=int, default=HEADLINE["order"])
    ap.add_argument("--bucket", type=int, default=HEADLINE["bucket"])
    ap.add_argument("--loc", type=float, default=HEADLINE["loc"],
                    help="local expansion of far cells: largest group half-diagonal "
                         "over cell distance (0 = off)")
    ap.add_argument("--nsamp", type=int, default=10,
                    help="TEMPORAL cadence of the timed loop (Nloop %% nsamp == 0)")
    ap.add_argument("--no-rdf", action="store_true",
                    help="time the loop without the per-step RDF pair counts")
    ap.add_argument("--workload", choices=["cloud", "ensemble"], default="cloud",
                    help="cloud: one N=1,048,576 cloud (headline); ensemble: 64 "
                         "independent clouds of uneven N in one handle")
    ap.add_argument("--clouds", type=int, default=64)
    ap.add_argument("--tune", action="store_true",
                    help="ensemble: autotune theta/eta/bucket/grid on the warm state")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the fixed-theta and plain-FP64 comparison arms")
    ap.add_argument("--fp64-thetas", default="0.35,0.25",
                    help="extra opening angles of the plain FP64 path (2 steps each) "
                         "for the equal-accuracy comparison")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the ensemble sub-record of the cloud workload")
    ap.add_argument("--ref-budget", type=float, default=100.0,
                    help="reference arm: stop timing whole steps after this many seconds")
    ap.add_argument("--ref-also-theta05", action="store_true",
                    help="reference arm: also time one whole Force call at the "
                         "reference's own theta = 0.5 with its own pair laws")
    ap.add_argument("--te", type=float, default=50.0)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--audit", type=int, default=16384,
                    help="targets of the FP64 direct-sum accuracy audit")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-stride", type=int, default=0,
                    help="walk every k-th target in the CPU sample (0: auto)")
    return ap.parse_args()


# --------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------- helpers ----
def make_workload(n, seed, te):
    from tree_b200 import cloud
    return cloud.make_cloud(n, seed=seed, te_k=te, ti_k=1e-3)


def workload_config(args, n):
    """The workload both arms run (no method keys): the same dict in the
    reference arm's line and in ours."""
    rdf = not args.no_rdf
    laws = "erf-Kelbg" if args.physics == "kelbg" else "reference (Coulomb + exp-screened e-i)"
    return {"workload": f"UCP cloud N={n} per GPU, T_e={args.te} K, T_i=1 mK, theta={args.theta}, "
                        f"{laws} pair laws, dt=1e-11 s, "
                        f"{'RDF pair counts every step, ' if rdf else ''}"
                        f"TEMPORAL sums every {args.nsamp} steps",
            "n_particles": n, "theta": args.theta, "te_k": args.te, "ti_k": 1e-3,
            "physics": args.physics, "dt_s": DT_S, "rdf": rdf, "nsamp": args.nsamp,
            "l2": "inputs larger than L2 (x,v,f 72 MB + trees >150 MB, rebuilt every step)"}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    return json.load(open(path)).get(kernel)


def fp_peak_tflops(sm_mhz, fp64):
    """CUDA-core peak of this GPU at the sampled SM clock: SMs x lanes x 2."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    lanes = 64 if fp64 else 128
    return sms * lanes * 2 * sm_mhz * 1e6 / 1e12


def oracle_params(args, theta=None, physics=None):
    import oracle
    from tree_b200 import units
    lam = units.kelbg_lambdas(args.te)
    phys = physics if physics is not None else (
        oracle.PHYS_KELBG if args.physics == "kelbg" else oracle.PHYS_REF)
    return oracle.make_params(theta=args.theta if theta is None else theta, rs=lam[1],
                              dx_ei=0.01, dx_ii=0.1, lambdas=lam, physics=phys)


def cpu_sample(c_state, args, stride):
    """Times the oracle on a state at the workload's configuration: full build
    of both trees, walk of every stride-th target; returns (particle-steps/s
    estimate, details)."""
    import oracle
    from tree_b200 import units
    p = oracle_params(args)
    x_el, x_ion = c_state["x_el"], c_state["x_ion"]
    n = len(x_el) + len(x_ion)
    t0 = time.perf_counter()
    r = oracle.force(x_el, x_ion, p, rdf=not args.no_rdf, stride=stride)
    wall = time.perf_counter() - t0
    st = r["stats"]
    xe, ve = x_el.copy(), c_state["v_el"].copy()
    t1 = time.perf_counter()
    oracle.kdk1(xe, ve, r["f_el"], units.dt_code(DT_S), units.M_ELECTRON_AMU)
    oracle.kdk2(ve, r["f_el"], units.dt_code(DT_S), units.M_ELECTRON_AMU)
    t_kdk = (time.perf_counter() - t1) * n / max(len(xe), 1)
    t_step = st["t_build"] + st["t_walk"] * stride + t_kdk
    return n / t_step, dict(t_build=st["t_build"], t_walk_sample=st["t_walk"],
                            t_kdk=t_kdk, stride=stride, wall=wall,
                            t_step_est=t_step)


def audit(tf, idx):
    """rms / max relative force error of the last computed forces against the
    FP64 O(N^2) direct sum on the GPU (tree_gpu_direct) at targets `idx`."""
    if idx is None:
        return None
    st = tf.get_state()
    fd, _ = tf.direct(idx)
    fw = np.vstack([st["f_el"], st["f_ion"]])[idx]
    err = np.linalg.norm(fw - fd, axis=1) / np.linalg.norm(fd, axis=1)
    return {"targets": int(len(idx)), "rms_rel_err": float(np.sqrt(np.mean(err**2))),
            "max_rel_err": float(err.max()),
            "judge": "FP64 O(N^2) direct sum on the GPU (tree_gpu_direct), same pair laws"}


def auto_stride(n):
    # about 3-6 s of sampled walking on ~8-100 host cores at N = 1M
    return max(1, int(round(n / 16384)))


def power_law(xs, ys):
    """Least-squares fit log y = a + b log x; returns (a, b)."""
    lx, ly = np.log(np.asarray(xs, float)), np.log(np.asarray(ys, float))
    b, a = np.polyfit(lx, ly, 1)
    return float(a), float(b)


def equal_accuracy(points, target=1e-4):
    """From (theta, rms, ms_per_step) of one path at several opening angles,
    the opening angle where rms reaches `target` and the time per step there,
    by power laws in theta fitted to the points (an extrapolation when the
    target lies outside them)."""
    pts = sorted(p for p in points if p[1] and p[1] > 0 and p[2] > 0)
    if len(pts) < 2:
        return None
    # the fit means something only where the error falls as theta shrinks
    # over every measured arm
    if any(b[1] <= a[1] for a, b in zip(pts, pts[1:])):
        return None
    th = [p[0] for p in pts]
    a_e, b_e = power_law(th, [p[1] for p in pts])
    a_t, b_t = power_law(th, [p[2] for p in pts])
    if b_e <= 0:
        return None
    theta_t = float(np.exp((np.log(target) - a_e) / b_e))
    if theta_t < 0.5 * min(th) or theta_t > 2.0 * max(th):
        return None  # too far outside the measured arms to report
    ms_t = float(np.exp(a_t + b_t * np.log(theta_t)))
    return {"target_rms": target, "theta": theta_t, "ms_per_step": ms_t,
            "rms_exponent": b_e, "time_exponent": b_t,
            "extrapolated": bool(theta_t < min(th) or theta_t > max(th)),
            "points": [{"theta": p[0], "rms": p[1], "ms_per_step": p[2]} for p in pts]}


# ------------------------------------------------------------- replicas ----
def max_over_ranks(value, dist):
    """The largest `value` over all ranks (the value itself without a process
    group): every rank reports the slowest replica's time."""
    if not dist:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(n_per_rank, world, steps, ms):
    """Particle-steps/s of all replicas together over a time of ms."""
    return n_per_rank * world * steps / (ms / 1e3)


# ----------------------------------------------------------- reference arm ----
def run_reference(args, rank, world):
    """Whole steps of the reference algorithm (the oracle) on the host cores:
    the initial force (Vinit, main.f90:777) untimed, then per step
    VVerletNotemp1 -> Force (with RDF) -> VVerletNotemp2 (main.f90:123-131),
    the kinetic sums on sample steps, until K steps or the time budget."""
    if rank != 0:
        return
    import oracle
    from tree_b200 import units
    flags = oracle.use_native()
    c = make_workload(args.n, args.seed, args.te)
    n = len(c.x_el) + len(c.x_ion)
    dt = units.dt_code(DT_S)
    p = oracle_params(args)
    rdf = not args.no_rdf
    xe, ve, xi, vi = c.x_el.copy(), c.v_el.copy(), c.x_ion.copy(), c.v_ion.copy()
    t0 = time.perf_counter()
    r = oracle.force(xe, xi, p, rdf=False)  # Vinit's force, untimed
    t_init = time.perf_counter() - t0
    fe, fi = r["f_el"], r["f_ion"]
    rei = np.zeros(oracle.NBINS, np.int64)
    rii = np.zeros(oracle.NBINS, np.int64)
    times, phases = [], []
    for k in range(max(args.steps, 1)):
        a = time.perf_counter()
        oracle.kdk1(xe, ve, fe, dt, units.M_ELECTRON_AMU)
        oracle.kdk1(xi, vi, fi, dt, units.M_ION_AMU)
        r = oracle.force(xe, xi, p, rdf=rdf)
        fe, fi = r["f_el"], r["f_ion"]
        if rdf:
            rei += r["rdf_ei"]
            rii += r["rdf_ii"]
        oracle.kdk2(ve, fe, dt, units.M_ELECTRON_AMU)
        oracle.kdk2(vi, fi, dt, units.M_ION_AMU)
        if args.nsamp > 0 and (k + 1) % args.nsamp == 0:
            oracle.ke(xe, ve, units.M_ELECTRON_AMU)
            oracle.ke(xi, vi, units.M_ION_AMU)
        times.append(time.perf_counter() - a)
        phases.append({"build_s": r["stats"]["t_build"], "walk_s": r["stats"]["t_walk"],
                       "n_m2p": r["stats"]["n_m2p"], "n_p2p": r["stats"]["n_p2p"]})
        if sum(times) >= args.ref_budget:
            break
    steps = len(times)
    total = sum(times)
    value = n * steps / total
    cores = oracle.max_threads()
    extra = None
    if args.ref_also_theta05:
        p05 = oracle_params(args, theta=0.5, physics=oracle.PHYS_REF)
        a = time.perf_counter()
        r05 = oracle.force(xe, xi, p05, rdf=rdf)
        t05 = time.perf_counter() - a
        extra = {"theta": 0.5, "pair_laws": "reference (Coulomb, exp-screened e-i, rs = lambda_ei)",
                 "force_s": t05, "particle_steps_per_s_force_only": n / t05,
                 "n_m2p": r05["stats"]["n_m2p"], "n_p2p": r05["stats"]["n_p2p"]}
    sample = (f"{steps} whole steps (VVerletNotemp1 + Force{' with RDF' if rdf else ''} + "
              f"VVerletNotemp2) of N={n} from the t = 0 cloud, after the untimed initial "
              f"force ({t_init:.1f} s); stopped at K={args.steps} steps or "
              f"{args.ref_budget:.0f} s of timed work")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * total / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian UCP cloud, electrons start on ions)",
        "config": workload_config(args, n),
        "method": {"algorithm": "reference (tree.f90:39-1133): per-species pointer octrees, "
                                "serial insertion, one-level moments, recursive per-target "
                                "walks (OpenMP, static schedule), FP64",
                   "mac": f"fixed theta = {args.theta}",
                   "implementation": f"oracle/tree_oracle.cpp (C++ restatement, {flags})"},
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "untimed": {"initial_force_s": t_init},
        "per_step_s": times, "per_step_phases": phases,
        "rdf_pairs_counted": int(rei.sum() + rii.sum()),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_theta0.5": extra,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours ----
def _timed_run(tf, stream, dt, steps, nsamp, rdf, dist):
    """tree_gpu_run of `steps` steps between CUDA events on the library's
    stream; returns (ms max over ranks, rdf pair count)."""
    import torch
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = tf.run(dt, steps, nsamp=nsamp, rdf=rdf)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    pairs = int(out[1][0].sum() + out[1][1].sum()) if rdf else None
    return max_over_ranks(e0.elapsed_time(e1), dist), pairs


def run_ours(args, rank, world, dist):
    import torch

    from tree_b200 import api, units
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    torch.cuda.init()
    prec = api.PREC_MIXED if args.precision == "mixed" else api.PREC_FP64
    phys = api.PHYS_KELBG if args.physics == "kelbg" else api.PHYS_REF
    mac = (api.MAC_LEARNED if args.mac == "learned" and args.precision == "mixed"
           else api.MAC_FIXED)
    cfg = api.Config(theta=args.theta, te=args.te, physics=phys, precision=prec,
                     mac=mac)
    dt = units.dt_code(DT_S)
    rdf = not args.no_rdf
    c = make_workload(args.n, args.seed + rank, args.te)
    n_el, n_ion = len(c.x_el), len(c.x_ion)
    n = n_el + n_ion
    stream = torch.cuda.Stream()
    tf = api.TreeForce(n_el, n_ion, cfg)
    tf.set_stream(stream.cuda_stream)
    if prec == api.PREC_MIXED:
        tf.set_tuning(args.bucket, 4, args.order)
        tf.set_local_expansion(args.loc)
        if mac == api.MAC_LEARNED:
            from tree_b200 import learned_mac
            params, stats, _ = learned_mac.load_model(order=args.order)
            tf.mac_set_model(params, stats)
            tf.mac_config(args.eta, 0.05, 0.9)
    tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
    warm = max(args.warmup, 3)
    tf.run(dt, warm, nsamp=args.nsamp, rdf=rdf)  # warm-up; e-i pairs separate
    torch.cuda.synchronize()
    st_warm = tf.get_state()  # every comparison arm starts from this state
    if dist:
        dist.barrier()

    # ---- timed region: device-resident state, K steps in one tree_gpu_run ----
    t_before = tf.timings()
    clocks = ClockSampler(dev)
    clocks.start()
    ms, rdf_pairs = _timed_run(tf, stream, dt, args.steps, args.nsamp, rdf, dist)
    clk = clocks.stop()
    t_after = tf.timings()
    value = whole_job_rate(n, world, args.steps, ms)
    walk_ms_sum = t_after.ms_walk - t_before.ms_walk
    build_ms_sum = t_after.ms_build - t_before.ms_build
    walk_ms = walk_ms_sum / args.steps
    build_ms = build_ms_sum / args.steps
    launches = t_after.launches - t_before.launches
    d_m2p = t_after.n_m2p_total - t_before.n_m2p_total
    d_p2p = t_after.n_p2p_total - t_before.n_p2p_total
    d_net = t_after.n_mac_net_total - t_before.n_mac_net_total
    d_loc = t_after.n_local_total - t_before.n_local_total

    # ---- accuracy audit of the last timed step: FP64 direct sum ----
    audit_idx = None
    if args.audit > 0:
        rng = np.random.default_rng(args.seed + 17)
        audit_idx = np.sort(rng.choice(n, min(args.audit, n), replace=False))
    accuracy = audit(tf, audit_idx)

    # ---- end to end: full state host->device, one step, state + RDF back ----
    e2e = None
    if not args.no_e2e:
        st = tf.get_state()
        pin = {k: torch.from_numpy(v).pin_memory() for k, v in st.items()}
        ptr = {k: v.data_ptr() for k, v in pin.items()}
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        k2 = max(1, min(args.steps, 5))
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k2):
            tf.load_state(ptr["x_el"], ptr["v_el"], ptr["f_el"], ptr["x_ion"],
                          ptr["v_ion"], ptr["f_ion"])
            tf.run(dt, 1, nsamp=1, rdf=rdf)
            tf.get_state_ptr(ptr["x_el"], ptr["v_el"], ptr["f_el"],
                             ptr["x_ion"], ptr["v_ion"], ptr["f_ion"])
        a1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(a0.elapsed_time(a1), dist)
        e2e = {"value": whole_job_rate(n, world, k2, ems), "unit": UNIT,
               "h2d_bytes_per_step": 72 * n,
               "d2h_bytes_per_step": 72 * n + SAMPLE_BYTES + (RDF_BYTES if rdf else 0),
               "steps": k2,
               "path": "tree_gpu_load_state(x,v,f pinned host) + tree_gpu_run(1 step, "
                       "TEMPORAL record, RDF) + tree_gpu_get_state(x,v,f pinned host)"}

    # ---- roofline of the dominant kernel (the walk), over the timed steps ----
    fp64 = prec == api.PREC_FP64
    fm2p = FLOPS_M2P_REF if fp64 else FLOPS_M2P_MIXED[args.order]
    fp2p = FLOPS_P2P_REF if fp64 else FLOPS_P2P_MIXED
    flops = d_m2p * fm2p + d_p2p * fp2p + (0 if fp64 else d_loc * FLOPS_LOCAL)
    achieved = flops / (walk_ms_sum / 1e3) / 1e12 if walk_ms_sum > 0 else 0.0
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak = fp_peak_tflops(sm_mhz, fp64)
    kname = "k_walk64" if fp64 else "k_walk_mixed"
    roofline = {"bound": "fp64" if fp64 else "fp32", "kernel": kname,
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "traffic": profile_traffic(kname),
                "peak_source": f"CUDA-core {'FP64' if fp64 else 'FP32'} peak = SMs x "
                               f"{64 if fp64 else 128} lanes x 2 x median SM clock "
                               f"{sm_mhz:.0f} MHz sampled during the run (the walk is "
                               "not a contraction; MEASURED_PEAKS.json has no CUDA-core figure)",
                "flops_per_launch": flops / args.steps, "walk_ms": walk_ms,
                "n_m2p_per_launch": d_m2p / args.steps, "n_p2p_per_launch": d_p2p / args.steps,
                "counts": f"interactions summed over the {args.steps} timed walks",
                "n_local_cells_per_launch": d_loc / args.steps,
                "flops_per_m2p": fm2p, "flops_per_p2p": fp2p, "flops_per_local_cell": FLOPS_LOCAL,
                "learned_mac_evals_per_launch": d_net / args.steps,
                "learned_mac_tensor_tflops": d_net * FLOPS_MLP / (walk_ms_sum / 1e3) / 1e12
                if walk_ms_sum > 0 else 0.0}
    pk, pk_kind = peaks()
    # build phase vs HBM: ~250 B per particle algorithmic
    build_bytes = 250 * n
    build_roof = {"bound": "hbm", "achieved": build_bytes / (build_ms / 1e3) / 1e9 if build_ms else None,
                  "peak": pk.get("hbm_gbs"), "unit": "GB/s",
                  "peak_source": pk_kind, "ms": build_ms,
                  "bytes_per_particle": 250}
    if build_roof["achieved"] and build_roof["peak"]:
        build_roof["frac"] = build_roof["achieved"] / build_roof["peak"]

    # ---- comparison arms: same warm state, same loop ----
    compare = None
    if not args.no_compare and prec == api.PREC_MIXED:
        compare = {"from": f"the state after the {warm} warm-up steps; every arm runs the "
                           f"same tree_gpu_run loop (RDF {'on' if rdf else 'off'}) and is "
                           f"audited after its last step"}
        arms = [(f"mixed_fixed_theta{th}", th, api.PREC_MIXED, args.steps)
                for th in FIXED_ARMS.get(args.order, FIXED_ARMS[3])]
        arms.append(("fp64_plain_theta0.5", 0.5, api.PREC_FP64, args.steps))
        sweep = [float(t) for t in args.fp64_thetas.split(",") if t.strip()]
        arms += [(f"fp64_plain_theta{th}", th, api.PREC_FP64, max(1, min(args.steps, 2)))
                 for th in sweep]
        for name, th, aprec, ksteps in arms:
            acfg = api.Config(theta=th, te=args.te, physics=phys, precision=aprec)
            with api.TreeForce(n_el, n_ion, acfg) as tc:
                tc.set_stream(stream.cuda_stream)
                if aprec == api.PREC_MIXED:
                    tc.set_tuning(args.bucket, 4, args.order)
                    tc.set_local_expansion(args.loc)
                tc.load_state(st_warm["x_el"], st_warm["v_el"], st_warm["f_el"],
                              st_warm["x_ion"], st_warm["v_ion"], st_warm["f_ion"])
                tb = tc.timings()
                cms, _ = _timed_run(tc, stream, dt, ksteps, args.nsamp, rdf, dist)
                ta = tc.timings()
                cms /= ksteps
                acc_c = audit(tc, audit_idx)
                compare[name] = {"theta": th, "steps": ksteps, "ms_per_step": cms,
                                 "walk_ms": (ta.ms_walk - tb.ms_walk) / ksteps,
                                 "particle_steps_per_s": n / (cms / 1e3),
                                 "rms_rel_err": acc_c and acc_c["rms_rel_err"],
                                 "max_rel_err": acc_c and acc_c["max_rel_err"],
                                 "n_m2p_per_step": (ta.n_m2p_total - tb.n_m2p_total) / ksteps,
                                 "n_local_cells_per_step": (ta.n_local_total - tb.n_local_total) / ksteps,
                                 "n_p2p_per_step": (ta.n_p2p_total - tb.n_p2p_total) / ksteps}
        ours_ms = ms / args.steps
        compare["headline_over_fp64_plain_theta0.5"] = (
            compare["fp64_plain_theta0.5"]["ms_per_step"] / ours_ms)
        fp64_pts = [(v["theta"], v["rms_rel_err"], v["ms_per_step"])
                    for k, v in compare.items()
                    if k.startswith("fp64_plain_theta") and isinstance(v, dict)]
        eq = equal_accuracy(fp64_pts, 1e-4)
        if eq is None and fp64_pts:
            # the plain path does not reach the bar on any arm it can run in
            # a bench (nor along a usable trend): its most accurate arm gives
            # a lower bound of the equal-accuracy speed-up
            best = min((p for p in fp64_pts if p[1]), key=lambda p: p[1], default=None)
            if best is not None:
                compare["fp64_plain_most_accurate_arm"] = {
                    "theta": best[0], "rms_rel_err": best[1], "ms_per_step": best[2],
                    "headline_over": best[2] / ours_ms,
                    "note": ("no plain FP64 arm reaches rms 1e-4 and its error does not fall "
                             "steadily with theta, so no equal-accuracy point is fitted; "
                             "this arm is still less accurate than the headline, so the "
                             "ratio is a lower bound")}
        if eq:
            eq["headline_over_fp64_at_equal_accuracy"] = eq["ms_per_step"] / ours_ms
            eq["note"] = ("plain FP64 fixed-theta path: rms error and time per step fitted as "
                          "power laws of theta over the measured arms, evaluated where the "
                          "rms reaches the headline's 1e-4 bar")
        compare["fp64_plain_equal_accuracy"] = eq

    # ---- ensemble of independent clouds (one handle, one launch per phase) ----
    ens_rec = None
    if not args.no_ensemble and prec == api.PREC_MIXED and mac == api.MAC_LEARNED:
        ens_rec = ensemble_record(args, stream, dist, world)

    # ---- CPU baseline (rank 0, N = 1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        flags = oracle.use_native()
        st = tf.get_state()
        stride = args.cpu_stride or auto_stride(n)
        v, det = cpu_sample(st, args, stride)
        cpu = {"value": v, "unit": UNIT, "cores": oracle.max_threads(),
               "kind": "port",
               "sample": f"oracle (reference algorithm, FP64, theta={args.theta}, "
                         f"{args.physics} pair laws{', RDF' if rdf else ''}) on the final "
                         f"state: full build + walk of every {stride}th target, walk time "
                         f"x{stride}; {flags}",
               "detail": det}

    tf.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if fp64 else "f32 (walk) + f64 (positions, Verlet, top cells)",
        "data": "synthetic (seeded Gaussian UCP cloud, electrons start on ions)",
        "config": workload_config(args, n),
        "method": {"precision": args.precision,
                   "mac": "learned" if mac == api.MAC_LEARNED else "fixed",
                   "eta": args.eta if mac == api.MAC_LEARNED else None,
                   "order": args.order, "bucket": args.bucket,
                   "local_expansion": args.loc if not fp64 else None,
                   "loop": "tree_gpu_run: CUDA-graph replay of the step body"},
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "clocks": clk, "e2e": e2e, "gpu_launches": launches,
        "phases_ms_per_step": {"build": build_ms, "walk": walk_ms,
                               "other": ms / args.steps - build_ms - walk_ms},
        "rdf_pairs_counted": rdf_pairs,
        "roofline": roofline, "roofline_build": build_roof,
        "accuracy": accuracy, "cpu_baseline": cpu, "compare": compare,
        "ensemble": ens_rec,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- ensemble ----
def ensemble_rms(ens, nclouds):
    """Per-cloud rms relative force error of the last forces against each
    cloud's own FP64 direct sum on 4,096 seeded targets."""
    f = ens.get_state()["f"]
    rms = []
    for cc in range(nclouds):
        a, b = int(ens.offsets[cc]), int(ens.offsets[cc + 1])
        t = np.sort(np.random.default_rng(cc).choice(b - a, min(4096, b - a), replace=False))
        fd, _ = ens.direct(cc, t)
        err = np.linalg.norm(f[a:b][t] - fd, axis=1) / np.linalg.norm(fd, axis=1)
        rms.append(float(np.sqrt(np.mean(err ** 2))))
    return rms


def ensemble_record(args, stream, dist, world, tune_it=False, compare_separate=False):
    """Independent clouds of uneven N (log-uniform in [8192, 131072]), peak
    densities log-uniform in [1e14, 1e16] m^-3, T_e uniform in [10, 200] K, in
    one handle: one build, one persistent walk launch and one integrator launch
    per step, replayed as CUDA graphs.  Optionally compared with the same clouds
    stepped one handle after another from the same state."""
    import torch

    from tree_b200 import api, cloud, learned_mac, tune, units
    dt = units.dt_code(DT_S)
    rank = int(os.environ.get("RANK", "0"))
    clouds, te, n0 = cloud.make_ensemble(args.clouds, seed=args.seed + rank)
    x, v, n_el, n_ion = cloud.pack_ensemble(clouds)
    n = len(x)
    phys = api.PHYS_KELBG if args.physics == "kelbg" else api.PHYS_REF
    setting = dict(ENSEMBLE_TUNED)
    mac = api.MAC_LEARNED if setting["eta"] > 0 else api.MAC_FIXED
    cfgs = [api.Config(theta=setting["theta"], te=float(t), physics=phys,
                       precision=api.PREC_MIXED, mac=mac) for t in te]
    params, stats, _ = learned_mac.load_model(order=setting["order"])
    ens = api.Ensemble(cfgs, n_el, n_ion)
    ens.set_stream(stream.cuda_stream)
    ens.set_tuning(setting["bucket"], setting["blocks_per_sm"], setting["order"])
    ens.mac_set_model(params, stats)
    ens.mac_config(setting["eta"], 0.05, 0.9)
    ens.set_state(x, v)
    # past the error transient of the first steps (electrons leaving their ions)
    ens.step(dt, max(args.warmup, 3) + 10)
    torch.cuda.synchronize()
    tuned = None
    if tune_it:
        order = args.order
        params, stats, _ = learned_mac.load_model(order=order)
        ens.set_tuning(setting["bucket"], setting["blocks_per_sm"], order)
        ens.mac_set_model(params, stats)
        space = [tune.Candidate(t, e, 8, order, g) for t in TUNE_THETAS.get(order, TUNE_THETAS[3])
                 for e in (0.0, 1e-5, 3e-5) for g in (2, 3)]
        best, trials = tune.autotune(ens, dt, space=space, target=1e-4, margin=0.8,
                                     audit=1024 * args.clouds, physics=phys,
                                     model=(params, stats))
        if best is not None:
            tuned = {**{k: getattr(best.cand, k) for k in ("theta", "eta", "bucket",
                                                           "order", "blocks_per_sm")},
                     "ms": best.ms, "rms": best.rms, "trials": len(trials)}
            setting = {k: tuned[k] for k in ENSEMBLE_TUNED}
    warm = ens.get_state()
    if dist:
        dist.barrier()
    t_before = ens.timings()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(dt, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    t_after = ens.timings()
    value = whole_job_rate(n, world, args.steps, ms)
    rms = ensemble_rms(ens, args.clouds)
    # end to end: cloud-major state host -> device, one step, state back
    pin = {k: torch.from_numpy(np.ascontiguousarray(warm[k])).pin_memory() for k in ("x", "v", "f")}
    k2 = max(1, min(args.steps, 5))
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(k2):
        ens.load_state(pin["x"].data_ptr(), pin["v"].data_ptr(), pin["f"].data_ptr())
        ens.step(dt, 1)
        ens.get_state_ptr(pin["x"].data_ptr(), pin["v"].data_ptr(), pin["f"].data_ptr())
    a1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(a0.elapsed_time(a1), dist) / k2
    fixed_arm = None
    if setting["eta"] > 0:
        # the same opening angle and order with the fixed test alone, from the
        # same warm state
        cand = tune.Candidate(setting["theta"], 0.0, setting["bucket"], setting["order"],
                              ENSEMBLE_FIXED_BPS)
        tune._apply(ens, cand, phys, 50.0, None)
        ens.load_state(warm["x"], warm["v"], warm["f"])
        ens.step(dt, 1)  # graph capture of this variant, untimed
        ens.load_state(warm["x"], warm["v"], warm["f"])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        ens.step(dt, args.steps)
        f1.record(stream)
        torch.cuda.synchronize()
        fms = max_over_ranks(f0.elapsed_time(f1), dist) / args.steps
        frms = ensemble_rms(ens, args.clouds)
        fixed_arm = {"theta": setting["theta"], "eta": 0.0, "blocks_per_sm": ENSEMBLE_FIXED_BPS,
                     "ms_per_step": fms, "value": whole_job_rate(n, world, 1, fms),
                     "rms_rel_err_max_cloud": max(frms),
                     "rms_rel_err_median_cloud": float(np.median(frms))}
    sep_ms = None
    if compare_separate:
        sep_ms = 0.0
        for cc in range(args.clouds):
            a, b = int(ens.offsets[cc]), int(ens.offsets[cc + 1])
            ne = int(n_el[cc])
            sl = {k: warm[k][a:b] for k in ("x", "v", "f")}
            cfg = api.Config(theta=setting["theta"], te=float(te[cc]), physics=phys,
                             precision=api.PREC_MIXED, mac=mac)
            with api.TreeForce(ne, b - a - ne, cfg) as tc:
                tc.set_stream(stream.cuda_stream)
                tc.set_tuning(setting["bucket"], setting["blocks_per_sm"], setting["order"])
                if setting["eta"] > 0:
                    tc.mac_set_model(params, stats)
                    tc.mac_config(setting["eta"], 0.05, 0.9)
                tc.load_state(sl["x"][:ne], sl["v"][:ne], sl["f"][:ne], sl["x"][ne:],
                              sl["v"][ne:], sl["f"][ne:])
                tc.step(dt, 1)
                tc.load_state(sl["x"][:ne], sl["v"][:ne], sl["f"][:ne], sl["x"][ne:],
                              sl["v"][ne:], sl["f"][ne:])
                s0 = torch.cuda.Event(enable_timing=True)
                s1 = torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                tc.step(dt, args.steps)
                s1.record(stream)
                torch.cuda.synchronize()
                sep_ms += max_over_ranks(s0.elapsed_time(s1), dist) / args.steps
    ens.close()
    return {
        "metric": f"particle-steps/s, ensemble of {args.clouds} independent clouds in one handle",
        "value": value, "unit": UNIT, "steps": args.steps, "ms_per_step": ms / args.steps,
        "workload": f"{args.clouds} clouds, N log-uniform in [8192, 131072] (total {n}), n0 "
                    f"log-uniform in [1e14, 1e16] m^-3, T_e uniform in [10, 200] K, T_i = 1 mK, "
                    f"dt = 1e-11 s; timed after {max(args.warmup, 3) + 10} steps; step loop "
                    f"without RDF (tree_gpu_run keeps RDF per single cloud only)",
        "n_particles": n, "setting": setting, "tuned_in_this_run": tuned,
        "clocks": clk, "gpu_launches": t_after.launches - t_before.launches,
        "phases_ms_per_step": {"build": (t_after.ms_build - t_before.ms_build) / args.steps,
                               "walk": (t_after.ms_walk - t_before.ms_walk) / args.steps},
        "accuracy": {"targets_per_cloud": 4096, "rms_rel_err_max_cloud": max(rms),
                     "rms_rel_err_median_cloud": float(np.median(rms)),
                     "per_cloud": [{"n": int(ens.offsets[cc + 1] - ens.offsets[cc]),
                                    "te_k": round(float(te[cc]), 2), "n0": float(n0[cc]),
                                    "rms": rms[cc]} for cc in range(args.clouds)]},
        "e2e": {"value": whole_job_rate(n, world, 1, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": 72 * n, "d2h_bytes_per_step": 72 * n},
        "fixed_theta_same_setting": fixed_arm,
        "separate_handles_ms_per_step": sep_ms,
        "one_launch_speedup": (sep_ms / (ms / args.steps)) if sep_ms else None,
    }


def run_ensemble(args, rank, world, dist):
    """The ensemble workload as the bench's own line."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    stream = torch.cuda.Stream()
    rec = ensemble_record(args, stream, dist, world, tune_it=args.tune,
                          compare_separate=not args.no_compare)
    if rank != 0:
        return
    line = {
        "metric": rec["metric"], "value": rec["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (walk) + f64 (positions, Verlet, top cells)",
        "data": "synthetic (seeded Gaussian UCP clouds, electrons start on ions)",
        "config": {"workload": rec["workload"], "n_particles": rec["n_particles"],
                   "l2": "inputs larger than L2"},
        "method": {"setting": rec["setting"], "tuned": rec["tuned_in_this_run"]},
        "clocks": rec["clocks"], "gpu_launches": rec["gpu_launches"],
        "phases_ms_per_step": rec["phases_ms_per_step"], "accuracy": rec["accuracy"],
        "e2e": rec["e2e"], "fixed_theta_same_setting": rec["fixed_theta_same_setting"],
        "separate_handles_ms_per_step": rec["separate_handles_ms_per_step"],
        "one_launch_speedup": rec["one_launch_speedup"],
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        # the reference arm runs on the host cores: gloo, no device
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        # rank 0 of the reference arm works for minutes while the others wait
        tdist.init_process_group(backend, timeout=datetime.timedelta(
            seconds=600 if backend == "nccl" else 1800))
        dist = tdist
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "ensemble":
            run_ensemble(args, rank, world, dist)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
