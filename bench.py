#!/usr/bin/env python
"""Benchmark of the TREE force path: particle-steps/s at N = 1,048,576.

One step = VVerletNotemp1 -> Force (octree build + upward pass + tree walk)
-> VVerletNotemp2, the loop body of main.f90:123-131 of hpjeonGIT/TREE, on a
seeded synthetic ultracold-plasma cloud (isotropic Gaussian of ions at peak
density 1e15 m^-3 with each electron starting on its ion, T_e = 50 K,
T_i = 1 mK, dt = 1e-11 s).  The inputs (positions, velocities, trees) are far
larger than the 126 MB L2 and every step rebuilds the trees from scratch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the CPU restatement of the reference algorithm
(pointer octree, serial insertion, recursive OpenMP walks in FP64 with the
reference pair laws) on the host cores, on a bounded sample of each step.
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

# Algorithmic flops per interaction, counted from the kernels' formulas
# (FMA = 2; divisions, square roots and exponentials count as one flop each).
FLOPS_M2P_REF = 194    # tree.f90:736-779 evaluated literally (FP64 path)
FLOPS_P2P_REF = 30     # leaf laws of tree.f90 / erf-Kelbg with the x^2>40 shortcut
FLOPS_M2P_MIXED = {2: 50, 3: 100}  # FP32 trace-free far field to quadrupole / octupole
FLOPS_P2P_MIXED = 24   # FP32 erf-Kelbg pair with hi/lo offsets
FLOPS_MLP = 2 * (16 * 64 + 64 * 64 + 64)  # one learned-MAC evaluation (BF16 mma + FP32)

# Headline configuration: mixed precision, learned MAC on top of theta = 0.30,
# octupole far field; chosen so the rms relative force error against the FP64
# direct sum stays below 1e-4 at this workload (measured by the accuracy audit
# below, which every run reports).
HEADLINE = dict(theta=0.30, eta=3e-5, order=3, bucket=8)


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
    ap.add_argument("--workload", choices=["cloud", "ensemble"], default="cloud",
                    help="cloud: one N=1,048,576 cloud (headline); ensemble: 64 "
                         "independent clouds of uneven N in one handle")
    ap.add_argument("--clouds", type=int, default=64)
    ap.add_argument("--tune", action="store_true",
                    help="ensemble: autotune theta/eta/bucket/grid on the warm state")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the fixed-theta and plain-FP64 comparison arms")
    ap.add_argument("--ref-theta", type=float, default=0.5,
                    help="opening angle of the reference CPU path (its own setting)")
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
    d = json.load(open(path)).get(kernel)
    return d


def fp_peak_tflops(sm_mhz, fp64):
    """CUDA-core peak of this GPU at the sampled SM clock: SMs x lanes x 2."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    lanes = 64 if fp64 else 128
    return sms * lanes * 2 * sm_mhz * 1e6 / 1e12


def cpu_sample(c_state, args, stride):
    """Times the oracle on the same state: full tree build, walk of every
    stride-th target; returns (particle-steps/s estimate, details)."""
    import oracle
    from tree_b200 import units
    lam = units.kelbg_lambdas(args.te)
    p = oracle.make_params(theta=args.ref_theta, rs=lam[1], lambdas=lam,
                           physics=oracle.PHYS_REF)
    x_el, x_ion = c_state["x_el"], c_state["x_ion"]
    n = len(x_el) + len(x_ion)
    t0 = time.perf_counter()
    r = oracle.force(x_el, x_ion, p, rdf=True, stride=stride)
    wall = time.perf_counter() - t0
    st = r["stats"]
    xe, ve = x_el.copy(), c_state["v_el"].copy()
    t1 = time.perf_counter()
    oracle.kdk1(xe, ve, r["f_el"], units.dt_code(1e-11), units.M_ELECTRON_AMU)
    oracle.kdk2(ve, r["f_el"], units.dt_code(1e-11), units.M_ELECTRON_AMU)
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
    if rank != 0:
        return
    import oracle
    c = make_workload(args.n, args.seed, args.te)
    rng = np.random.Generator(np.random.Philox(args.seed + 1))
    # the state a few steps after t = 0: each electron near its ion
    state = dict(x_el=c.x_ion + rng.standard_normal(c.x_ion.shape) * 0.3,
                 x_ion=c.x_ion, v_el=c.v_el)
    stride = args.cpu_stride or auto_stride(args.n)
    for _ in range(args.warmup):
        cpu_sample(state, args, stride * 4)
    vals, det = [], None
    for _ in range(args.steps):
        v, det = cpu_sample(state, args, stride)
        vals.append(v)
    value = float(np.median(vals))
    cores = oracle.max_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * args.n / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian UCP cloud)",
        "config": {"workload": f"UCP cloud N={args.n}, T_e={args.te} K, T_i=1 mK, "
                               f"dt=1e-11 s; reference algorithm at its own opening angle "
                               f"theta={args.ref_theta} (less accurate than the GPU arm's "
                               f"rms <= 1e-4), reference pair laws, FP64",
                   "n_particles": args.n, "theta": args.ref_theta},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                         "kind": "port",
                         "sample": f"full build of both trees + walk of every "
                                   f"{stride}th target, walk time x{stride}; "
                                   f"median of {args.steps} samples",
                         "detail": det},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours ----
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
    dt = units.dt_code(1e-11)
    c = make_workload(args.n, args.seed + rank, args.te)
    n_el, n_ion = len(c.x_el), len(c.x_ion)
    n = n_el + n_ion
    stream = torch.cuda.Stream()
    tf = api.TreeForce(n_el, n_ion, cfg)
    tf.set_stream(stream.cuda_stream)
    if prec == api.PREC_MIXED:
        tf.set_tuning(args.bucket, 4, args.order)
        if mac == api.MAC_LEARNED:
            from tree_b200 import learned_mac
            params, stats, _ = learned_mac.load_model()
            tf.mac_set_model(params, stats)
            tf.mac_config(args.eta, 0.05, 0.9)
    tf.set_state(c.x_el, c.v_el, c.x_ion, c.v_ion)
    tf.step(dt, max(args.warmup, 3))  # warm-up; e-i pairs separate
    torch.cuda.synchronize()
    st_warm = tf.get_state()  # every comparison arm starts from this state
    if dist:
        dist.barrier()

    # ---- timed region: device-resident state, K steps in one call ----
    t_before = tf.timings()
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    diag = tf.step(dt, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    t_after = tf.timings()
    value = whole_job_rate(n, world, args.steps, ms)
    walk_ms = (t_after.ms_walk - t_before.ms_walk) / args.steps
    build_ms = (t_after.ms_build - t_before.ms_build) / args.steps
    launches = t_after.launches - t_before.launches
    n_m2p, n_p2p = t_after.n_m2p, t_after.n_p2p
    n_net = t_after.n_mac_net

    # ---- accuracy audit of the last timed step: FP64 direct sum ----
    audit_idx = None
    if args.audit > 0:
        rng = np.random.default_rng(args.seed + 17)
        audit_idx = np.sort(rng.choice(n, min(args.audit, n), replace=False))
    accuracy = audit(tf, audit_idx)

    # ---- end to end: full state host->device, one step, state back ----
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
            tf.step(dt, 1)
            tf.get_state_ptr(ptr["x_el"], ptr["v_el"], ptr["f_el"],
                             ptr["x_ion"], ptr["v_ion"], ptr["f_ion"])
        a1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(a0.elapsed_time(a1), dist)
        e2e = {"value": whole_job_rate(n, world, k2, ems), "unit": UNIT,
               "h2d_bytes_per_step": 72 * n, "d2h_bytes_per_step": 72 * n,
               "steps": k2,
               "path": "tree_gpu_load_state(x,v,f pinned host) + tree_gpu_step(1) "
                       "+ tree_gpu_get_state(x,v,f pinned host)"}

    # ---- roofline of the dominant kernel (the walk) ----
    fp64 = prec == api.PREC_FP64
    fm2p = FLOPS_M2P_REF if fp64 else FLOPS_M2P_MIXED[args.order]
    fp2p = FLOPS_P2P_REF if fp64 else FLOPS_P2P_MIXED
    flops = n_m2p * fm2p + n_p2p * fp2p
    achieved = flops / (walk_ms / 1e3) / 1e12 if walk_ms > 0 else 0.0
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
                "flops_per_launch": flops, "walk_ms": walk_ms,
                "n_m2p": n_m2p, "n_p2p": n_p2p,
                "flops_per_m2p": fm2p, "flops_per_p2p": fp2p,
                "learned_mac_evals": n_net,
                "learned_mac_tensor_tflops": n_net * FLOPS_MLP / (walk_ms / 1e3) / 1e12 if walk_ms > 0 else 0.0}
    pk, pk_kind = peaks()
    # build phase vs HBM: ~250 B per particle algorithmic
    build_bytes = 250 * n
    build_roof = {"bound": "hbm", "achieved": build_bytes / (build_ms / 1e3) / 1e9 if build_ms else None,
                  "peak": pk.get("hbm_gbs"), "unit": "GB/s",
                  "peak_source": pk_kind, "ms": build_ms,
                  "bytes_per_particle": 250}
    if build_roof["achieved"] and build_roof["peak"]:
        build_roof["frac"] = build_roof["achieved"] / build_roof["peak"]

    # ---- comparison arms: same warm state, same number of steps ----
    compare = None
    if not args.no_compare and prec == api.PREC_MIXED:
        compare = {"from": f"the state after the {max(args.warmup, 3)} warm-up steps, "
                           f"{args.steps} steps each, audit after the last"}
        arms = [(f"mixed_fixed_theta{th}", api.Config(theta=th, te=args.te, physics=phys,
                                                      precision=api.PREC_MIXED))
                for th in (0.30, 0.32, 0.35)]
        arms.append(("fp64_plain_theta0.5", api.Config(theta=0.5, te=args.te, physics=phys,
                                                       precision=api.PREC_FP64)))
        for name, acfg in arms:
            with api.TreeForce(n_el, n_ion, acfg) as tc:
                tc.set_stream(stream.cuda_stream)
                if acfg.precision == api.PREC_MIXED:
                    tc.set_tuning(args.bucket, 4, args.order)
                tc.load_state(st_warm["x_el"], st_warm["v_el"], st_warm["f_el"],
                              st_warm["x_ion"], st_warm["v_ion"], st_warm["f_ion"])
                torch.cuda.synchronize()
                tb = tc.timings()
                b0 = torch.cuda.Event(enable_timing=True)
                b1 = torch.cuda.Event(enable_timing=True)
                b0.record(stream)
                tc.step(dt, args.steps)
                b1.record(stream)
                torch.cuda.synchronize()
                ta = tc.timings()
                cms = max_over_ranks(b0.elapsed_time(b1), dist) / args.steps
                acc_c = audit(tc, audit_idx)
                compare[name] = {"theta": acfg.theta, "ms_per_step": cms,
                                 "walk_ms": (ta.ms_walk - tb.ms_walk) / args.steps,
                                 "particle_steps_per_s": n / (cms / 1e3),
                                 "rms_rel_err": acc_c and acc_c["rms_rel_err"],
                                 "max_rel_err": acc_c and acc_c["max_rel_err"],
                                 "n_m2p_last": ta.n_m2p, "n_p2p_last": ta.n_p2p}
        compare["headline_over_fp64_plain"] = (value / world /
                                               compare["fp64_plain_theta0.5"]["particle_steps_per_s"])

    # ---- CPU baseline (rank 0, N = 1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        st = tf.get_state()
        stride = args.cpu_stride or auto_stride(n)
        v, det = cpu_sample(st, args, stride)
        cpu = {"value": v, "unit": UNIT, "cores": oracle.max_threads(),
               "kind": "port",
               "sample": f"oracle REF1 (reference algorithm, FP64, reference pair laws, "
                         f"theta={args.ref_theta}) on the final state: full build + walk "
                         f"of every {stride}th target, walk time x{stride}",
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
        "config": {"workload": f"UCP cloud N={n} per GPU, T_e={args.te} K, T_i=1 mK, "
                               f"theta={args.theta}, dt=1e-11 s",
                   "n_particles": n, "theta": args.theta, "te_k": args.te,
                   "physics": args.physics, "precision": args.precision,
                   "mac": "learned" if mac == api.MAC_LEARNED else "fixed",
                   "eta": args.eta if mac == api.MAC_LEARNED else None,
                   "order": args.order, "bucket": args.bucket,
                   "l2": "inputs larger than L2 (x,v,f 72 MB + trees >150 MB, rebuilt every step)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk, "e2e": e2e, "gpu_launches": launches,
        "phases_ms_per_step": {"build": build_ms, "walk": walk_ms,
                               "other": ms / args.steps - build_ms - walk_ms},
        "roofline": roofline, "roofline_build": build_roof,
        "accuracy": accuracy, "cpu_baseline": cpu, "compare": compare,
        "diag": {"epot_e": diag.epot_e, "epot_i": diag.epot_i,
                 "mv2_el": diag.mv2_el, "mv2_ion": diag.mv2_ion},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- ensemble ----
def run_ensemble(args, rank, world, dist):
    """Independent clouds of uneven N (log-uniform in [8192, 131072]), peak
    densities log-uniform in [1e14, 1e16] m^-3, T_e uniform in [10, 200] K, in
    one handle: one build, one persistent walk launch and one integrator launch
    per step, replayed as CUDA graphs.  Compared with the same clouds stepped
    one handle after another from the same state."""
    import torch

    from tree_b200 import api, cloud, learned_mac, tune, units
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    dt = units.dt_code(1e-11)
    clouds, te, n0 = cloud.make_ensemble(args.clouds, seed=args.seed + rank)
    x, v, n_el, n_ion = cloud.pack_ensemble(clouds)
    n = len(x)
    phys = api.PHYS_KELBG if args.physics == "kelbg" else api.PHYS_REF
    mac = api.MAC_LEARNED if args.mac == "learned" else api.MAC_FIXED
    cfgs = [api.Config(theta=args.theta, te=float(t), physics=phys,
                       precision=api.PREC_MIXED, mac=mac) for t in te]
    params, stats, _ = learned_mac.load_model()
    stream = torch.cuda.Stream()
    ens = api.Ensemble(cfgs, n_el, n_ion)
    ens.set_stream(stream.cuda_stream)
    ens.set_tuning(args.bucket, 4, args.order)
    ens.mac_set_model(params, stats)
    ens.mac_config(args.eta, 0.05, 0.9)
    ens.set_state(x, v)
    ens.step(dt, max(args.warmup, 3))
    torch.cuda.synchronize()
    tuned = None
    if args.tune:
        # the force error grows while the electrons leave their ions (about
        # ten steps of 1e-11 s): tune on a state past that transient
        ens.step(dt, 10)
        space = [tune.Candidate(t, e, 8, 3, g) for t in (0.20, 0.22, 0.24, 0.26, 0.28, 0.30)
                 for e in (0.0, 3e-6, 1e-5, 3e-5) for g in (3, 4)]
        # 1024 audited targets per cloud; margin 0.8 leaves room for the state
        # to drift during the timed steps
        best, trials = tune.autotune(ens, dt, space=space, target=1e-4, margin=0.8,
                                     audit=1024 * args.clouds, physics=phys,
                                     model=(params, stats))
        if best is not None:
            tuned = {**{k: getattr(best.cand, k) for k in ("theta", "eta", "bucket",
                                                           "order", "blocks_per_sm")},
                     "ms": best.ms, "rms": best.rms, "trials": len(trials)}
    warm = ens.get_state()
    if dist:
        dist.barrier()
    t_before = ens.timings()
    clocks = ClockSampler(dev)
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
    # per-cloud accuracy against each cloud's own FP64 direct sum
    f = ens.get_state()["f"]
    rms = []
    for c in range(args.clouds):
        a, b = int(ens.offsets[c]), int(ens.offsets[c + 1])
        t = np.sort(np.random.default_rng(c).choice(b - a, min(4096, b - a), replace=False))
        fd, _ = ens.direct(c, t)
        err = np.linalg.norm(f[a:b][t] - fd, axis=1) / np.linalg.norm(fd, axis=1)
        rms.append(float(np.sqrt(np.mean(err ** 2))))
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
    # the same clouds, one handle after another, from the same warm state
    sep_ms = None
    if not args.no_compare:
        tb = ens.timings()
        sep_ms = 0.0
        for c in range(args.clouds):
            a, b = int(ens.offsets[c]), int(ens.offsets[c + 1])
            ne = int(n_el[c])
            sl = {k: warm[k][a:b] for k in ("x", "v", "f")}
            cfg = api.Config(theta=ens.config.theta, te=float(te[c]), physics=phys,
                             precision=api.PREC_MIXED, mac=ens.config.mac)
            with api.TreeForce(ne, b - a - ne, cfg) as tc:
                tc.set_stream(stream.cuda_stream)
                tc.set_tuning(args.bucket, 4, args.order)
                eta_c = args.eta if tuned is None else tuned["eta"]
                if eta_c > 0:
                    tc.mac_set_model(params, stats)
                    tc.mac_config(eta_c, 0.05, 0.9)
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
    if rank != 0:
        return
    walk_ms = (t_after.ms_walk - t_before.ms_walk) / args.steps
    build_ms = (t_after.ms_build - t_before.ms_build) / args.steps
    line = {
        "metric": f"particle-steps/s, ensemble of {args.clouds} independent clouds in one handle",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (walk) + f64 (positions, Verlet, top cells)",
        "data": "synthetic (seeded Gaussian UCP clouds, electrons start on ions)",
        "config": {"workload": f"{args.clouds} clouds, N log-uniform in [8192, 131072] "
                               f"(total {n}), n0 log-uniform in [1e14, 1e16] m^-3, "
                               f"T_e uniform in [10, 200] K, T_i = 1 mK, dt = 1e-11 s",
                   "n_particles": n, "theta": ens.config.theta,
                   "mac": "learned" if ens.config.mac == api.MAC_LEARNED else "fixed",
                   "eta": args.eta if tuned is None else tuned["eta"], "tuned": tuned,
                   "l2": "inputs larger than L2"},
        "clocks": clk, "gpu_launches": t_after.launches - t_before.launches,
        "phases_ms_per_step": {"build": build_ms, "walk": walk_ms},
        "accuracy": {"targets_per_cloud": 4096, "rms_rel_err_max_cloud": max(rms),
                     "rms_rel_err_median_cloud": float(np.median(rms)),
                     "per_cloud": [{"n": int(ens.offsets[c + 1] - ens.offsets[c]),
                                    "te_k": round(float(te[c]), 2), "n0": float(n0[c]),
                                    "rms": rms[c]} for c in range(args.clouds)]},
        "e2e": {"value": whole_job_rate(n, world, 1, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": 72 * n, "d2h_bytes_per_step": 72 * n},
        "separate_handles_ms_per_step": sep_ms,
        "one_launch_speedup": (sep_ms / (ms / args.steps)) if sep_ms else None,
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
        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
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
