"""Python mirror of the force boundary (ctypes over libtree_b200.so).

The reference's interface is ``SUBROUTINE Force(NS, qel, qion, param, ttime)``
(main.f90:506-701 of hpjeonGIT/TREE) plus the velocity-Verlet calls of its step
loop (main.f90:125-131, vverlet.f90:9-112).  ``TreeForce.force`` mirrors Force:
positions in, forces and potential energies out, RDF histograms accumulated.
``TreeForce.set_state / step / get_state`` mirror the step loop with the state
resident on the GPU.  Every call goes through the C ABI of include/tree_gpu.h;
there is no CPU fallback: a missing library raises ImportError.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import units

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtree_b200.so")

OK = 0
ERR = {-1: "ARG", -2: "DEPTH", -3: "NONFINITE", -4: "CAPACITY", -5: "CUDA",
       -6: "WALK", -7: "STATE"}
PHYS_REF, PHYS_KELBG = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
MAC_FIXED, MAC_LEARNED = 0, 1
RDF_BINS = 10001

# Every symbol include/tree_gpu.h declares.
EXPORTS = ("tree_gpu_create", "tree_gpu_set_params", "tree_gpu_force",
           "tree_gpu_set_state", "tree_gpu_load_state", "tree_gpu_step",
           "tree_gpu_run", "tree_gpu_set_graphs", "tree_gpu_get_nloop",
           "tree_gpu_get_state", "tree_gpu_direct", "tree_gpu_direct_static",
           "tree_gpu_tree_dump", "tree_gpu_net_dump", "tree_gpu_set_stream", "tree_gpu_set_tuning",
           "tree_gpu_set_local_expansion",
           "tree_gpu_mac_collect", "tree_gpu_mac_samples", "tree_gpu_mac_clear",
           "tree_gpu_mac_train", "tree_gpu_mac_set_model",
           "tree_gpu_mac_get_model", "tree_gpu_mac_config", "tree_gpu_mlp_grad",
           "tree_gpu_mlp_infer", "tree_gpu_timings", "tree_gpu_last_error",
           "tree_gpu_destroy", "tree_gpu_version", "tree_gpu_ensemble_create",
           "tree_gpu_ensemble_set_state", "tree_gpu_ensemble_load_state",
           "tree_gpu_ensemble_get_state", "tree_gpu_ensemble_sums",
           "tree_gpu_ensemble_direct")


class Params(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_double), ("rs", ctypes.c_double),
                ("te", ctypes.c_double), ("xm_el", ctypes.c_double),
                ("xm_ion", ctypes.c_double), ("dx_ei", ctypes.c_double),
                ("dx_ii", ctypes.c_double), ("physics", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("mac", ctypes.c_int32),
                ("group", ctypes.c_int32)]


class Diag(ctypes.Structure):
    _fields_ = [("epot_e", ctypes.c_double), ("epot_i", ctypes.c_double),
                ("mv2_el", ctypes.c_double), ("mv2_ion", ctypes.c_double),
                ("rad_el", ctypes.c_double), ("rad_ion", ctypes.c_double),
                ("steps_done", ctypes.c_int64)]


class Sample(ctypes.Structure):
    _fields_ = [("nloop", ctypes.c_int64), ("epot_e", ctypes.c_double),
                ("epot_i", ctypes.c_double), ("mv2_el", ctypes.c_double),
                ("mv2_ion", ctypes.c_double), ("rad_el", ctypes.c_double),
                ("rad_ion", ctypes.c_double)]


class Timing(ctypes.Structure):
    _fields_ = [("ms_build", ctypes.c_double), ("ms_walk", ctypes.c_double),
                ("ms_kdk", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("n_m2p", ctypes.c_int64), ("n_p2p", ctypes.c_int64),
                ("n_nodes", ctypes.c_int64), ("calls", ctypes.c_int64),
                ("launches", ctypes.c_int64), ("n_mac_net", ctypes.c_int64),
                ("n_mac_fallback", ctypes.c_int64), ("n_m2p_total", ctypes.c_int64),
                ("n_p2p_total", ctypes.c_int64), ("n_mac_net_total", ctypes.c_int64),
                ("n_local", ctypes.c_int64), ("n_local_total", ctypes.c_int64)]


class TreeGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tree_gpu error {code} ({ERR.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libtree_b200.so; raises ImportError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} not built: run `python -m tree_b200.build`")
    L = ctypes.CDLL(path)
    vp, dp, lp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
    L.tree_gpu_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int64,
                                  ctypes.c_int64, ctypes.POINTER(vp)]
    L.tree_gpu_set_params.argtypes = [vp, ctypes.POINTER(Params)]
    L.tree_gpu_force.argtypes = [vp, dp, dp, dp, dp, dp, dp, lp, lp]
    L.tree_gpu_set_state.argtypes = [vp, dp, dp, dp, dp]
    L.tree_gpu_load_state.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    L.tree_gpu_step.argtypes = [vp, ctypes.c_double, ctypes.c_int32,
                                ctypes.POINTER(Diag)]
    L.tree_gpu_run.argtypes = [vp, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                               ctypes.POINTER(Sample), ctypes.c_int32,
                               ctypes.POINTER(ctypes.c_int32), lp, lp]
    L.tree_gpu_set_graphs.argtypes = [vp, ctypes.c_int32]
    L.tree_gpu_get_nloop.argtypes = [vp, lp]
    L.tree_gpu_get_state.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    L.tree_gpu_tree_dump.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, dp,
                                     dp, dp, ctypes.POINTER(ctypes.c_int32),
                                     lp, lp, lp]
    L.tree_gpu_net_dump.argtypes = [vp, ctypes.c_int64, dp, dp, lp, lp,
                                    ctypes.POINTER(ctypes.c_int32), lp, dp, lp]
    L.tree_gpu_direct.argtypes = [vp, lp, ctypes.c_int64, dp, dp]
    L.tree_gpu_direct_static.argtypes = [vp, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.POINTER(Params), vp,
                                         ctypes.c_int64, vp, vp, vp]
    L.tree_gpu_set_stream.argtypes = [vp, vp]
    L.tree_gpu_set_tuning.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.tree_gpu_set_local_expansion.argtypes = [vp, ctypes.c_double]
    fp = ctypes.POINTER(ctypes.c_float)
    L.tree_gpu_mac_collect.argtypes = [vp, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, ctypes.c_float,
                                       ctypes.c_uint64, ctypes.c_int64, lp]
    L.tree_gpu_mac_samples.argtypes = [vp, fp, fp, fp, ctypes.c_int64, lp]
    L.tree_gpu_mac_clear.argtypes = [vp]
    L.tree_gpu_mac_train.argtypes = [vp, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_float, ctypes.c_float,
                                     ctypes.c_uint64, fp]
    L.tree_gpu_mac_set_model.argtypes = [vp, fp, fp]
    L.tree_gpu_mac_get_model.argtypes = [vp, fp, fp]
    L.tree_gpu_mac_config.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    L.tree_gpu_mlp_grad.argtypes = [fp, fp, ctypes.c_int64, fp, ctypes.c_float, fp, fp]
    L.tree_gpu_mlp_infer.argtypes = [fp, ctypes.c_int64, fp, fp, fp]
    L.tree_gpu_timings.argtypes = [vp, ctypes.POINTER(Timing)]
    L.tree_gpu_last_error.argtypes = [vp]
    L.tree_gpu_last_error.restype = ctypes.c_char_p
    L.tree_gpu_destroy.argtypes = [vp]
    L.tree_gpu_version.restype = ctypes.c_char_p
    L.tree_gpu_ensemble_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, lp, lp,
                                           ctypes.POINTER(vp)]
    L.tree_gpu_ensemble_set_state.argtypes = [vp, dp, dp]
    L.tree_gpu_ensemble_load_state.argtypes = [vp, dp, dp, dp]
    L.tree_gpu_ensemble_get_state.argtypes = [vp, dp, dp, dp]
    L.tree_gpu_ensemble_sums.argtypes = [vp, dp]
    L.tree_gpu_ensemble_direct.argtypes = [vp, ctypes.c_int32, lp, ctypes.c_int64, dp, dp]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or ctypes.c_int
    _lib = L
    return L


MLP_PARAMS = 5313
MLP_STATS = 72


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_grad(X, y, params, tau=0.9):
    """Device gradient of the mean pinball loss (tree_gpu_mlp_grad)."""
    L = load_library()
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    rc = L.tree_gpu_mlp_grad(_fp(X), _fp(y), len(X), _fp(p), tau, _fp(g), _fp(loss))
    if rc != OK:
        raise TreeGpuError(rc, "tree_gpu_mlp_grad")
    return float(loss[0]), g


def mlp_infer(X, params, stats):
    """Device inference of the packed network on raw features."""
    L = load_library()
    X = np.ascontiguousarray(X, np.float32)
    y = np.zeros(len(X), np.float32)
    rc = L.tree_gpu_mlp_infer(_fp(X), len(X), _fp(np.ascontiguousarray(params, np.float32)),
                              _fp(np.ascontiguousarray(stats, np.float32)), _fp(y))
    if rc != OK:
        raise TreeGpuError(rc, "tree_gpu_mlp_infer")
    return y


def _dp(a):
    if a is None:
        return None
    if isinstance(a, int):  # raw address (e.g. pinned host memory)
        return ctypes.cast(a, ctypes.POINTER(ctypes.c_double))
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c3(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, 3))


@dataclass
class Config:
    """Arguments of the force path (the fields of TYPE(PM)/TYPE(NM) the walk
    reads).  rs defaults to lambda_ei, the recommended REF screening length."""
    theta: float = 0.5
    te: float = 50.0
    rs: float | None = None
    xm_el: float = units.M_ELECTRON_AMU
    xm_ion: float = units.M_ION_AMU
    dx_ei: float = 0.01
    dx_ii: float = 0.1
    physics: int = PHYS_REF
    precision: int = PREC_FP64
    mac: int = MAC_FIXED
    group: int = 0

    def to_c(self) -> Params:
        rs = self.rs if self.rs is not None else units.kelbg_lambdas(
            self.te, self.xm_el, self.xm_ion)[1]
        return Params(self.theta, rs, self.te, self.xm_el, self.xm_ion,
                      self.dx_ei, self.dx_ii, self.physics, self.precision,
                      self.mac, self.group)


class TreeForce:
    """One device-resident force path for n_el electrons and n_ion ions."""

    def __init__(self, n_el: int, n_ion: int, config: Config | None = None):
        self.lib = load_library()
        self.n_el, self.n_ion = int(n_el), int(n_ion)
        self.config = config or Config()
        self._p = self.config.to_c()
        h = ctypes.c_void_p()
        rc = self.lib.tree_gpu_create(ctypes.byref(self._p), self.n_el,
                                      self.n_ion, ctypes.byref(h))
        if rc != OK:
            raise TreeGpuError(rc, "tree_gpu_create failed")
        self.h = h

    def _check(self, rc):
        if rc != OK:
            msg = self.lib.tree_gpu_last_error(self.h)
            raise TreeGpuError(rc, msg.decode() if msg else "")

    def set_config(self, config: Config):
        self.config = config
        self._p = config.to_c()
        self._check(self.lib.tree_gpu_set_params(self.h, ctypes.byref(self._p)))

    def force(self, x_el, x_ion, rdf_ei=None, rdf_ii=None):
        """Mirror of Force: returns (f_el, f_ion, epot_e, epot_i); rdf_* are
        int64 arrays of 10001 bins that are accumulated in place."""
        x_el, x_ion = _c3(x_el), _c3(x_ion)
        assert len(x_el) == self.n_el and len(x_ion) == self.n_ion
        f_el = np.empty_like(x_el)
        f_ion = np.empty_like(x_ion)
        ee = ctypes.c_double()
        ei = ctypes.c_double()
        lp = ctypes.POINTER(ctypes.c_int64)
        for r in (rdf_ei, rdf_ii):
            if r is not None:
                assert r.dtype == np.int64 and r.size == RDF_BINS and r.flags.c_contiguous
        self._check(self.lib.tree_gpu_force(
            self.h, _dp(x_el), _dp(x_ion), _dp(f_el), _dp(f_ion),
            ctypes.byref(ee), ctypes.byref(ei),
            rdf_ei.ctypes.data_as(lp) if rdf_ei is not None else None,
            rdf_ii.ctypes.data_as(lp) if rdf_ii is not None else None))
        return f_el, f_ion, ee.value, ei.value

    def set_state(self, x_el, v_el, x_ion, v_ion):
        x_el, v_el, x_ion, v_ion = map(_c3, (x_el, v_el, x_ion, v_ion))
        self._check(self.lib.tree_gpu_set_state(self.h, _dp(x_el), _dp(v_el),
                                                _dp(x_ion), _dp(v_ion)))

    def set_state_ptr(self, x_el, v_el, x_ion, v_ion):
        """set_state from raw host addresses (pinned buffers)."""
        self._check(self.lib.tree_gpu_set_state(self.h, _dp(x_el), _dp(v_el),
                                                _dp(x_ion), _dp(v_ion)))

    def load_state(self, x_el, v_el, f_el, x_ion, v_ion, f_ion):
        """Full state in (no force evaluation); arrays or raw host addresses."""
        conv = (lambda a: a) if isinstance(x_el, int) else _c3
        args = [conv(a) for a in (x_el, v_el, f_el, x_ion, v_ion, f_ion)]
        self._check(self.lib.tree_gpu_load_state(self.h, *[_dp(a) for a in args]))

    def step(self, dt: float, nsteps: int = 1) -> Diag:
        d = Diag()
        self._check(self.lib.tree_gpu_step(self.h, dt, nsteps, ctypes.byref(d)))
        return d

    def run(self, dt: float, nsteps: int, nsamp: int = 0, rdf: bool = False):
        """The step loop with the reference's sampling cadence.  Returns the
        sample records (a structured array) and, with rdf, the (rdf_ei,
        rdf_ii) pair counts accumulated over every step of the call."""
        ns = max(1, nsteps // nsamp + 1) if nsamp > 0 else 1
        buf = (Sample * ns)()
        cnt = ctypes.c_int32(0)
        r_ei = np.zeros(RDF_BINS, np.int64) if rdf else None
        r_ii = np.zeros(RDF_BINS, np.int64) if rdf else None
        lp = ctypes.POINTER(ctypes.c_int64)
        self._check(self.lib.tree_gpu_run(
            self.h, dt, nsteps, nsamp, buf, ns, ctypes.byref(cnt),
            r_ei.ctypes.data_as(lp) if rdf else None,
            r_ii.ctypes.data_as(lp) if rdf else None))
        dtype = np.dtype([(name, np.int64 if name == "nloop" else np.float64)
                          for name, _ in Sample._fields_])
        rec = np.zeros(cnt.value, dtype)
        for k in range(cnt.value):
            for name, _ in Sample._fields_:
                rec[name][k] = getattr(buf[k], name)
        return (rec, (r_ei, r_ii)) if rdf else rec

    def set_graphs(self, enable: bool):
        self._check(self.lib.tree_gpu_set_graphs(self.h, 1 if enable else 0))

    def nloop(self) -> int:
        v = ctypes.c_int64(0)
        self._check(self.lib.tree_gpu_get_nloop(self.h, ctypes.byref(v)))
        return v.value

    def get_state(self):
        x_el = np.empty((self.n_el, 3))
        v_el = np.empty_like(x_el)
        f_el = np.empty_like(x_el)
        x_ion = np.empty((self.n_ion, 3))
        v_ion = np.empty_like(x_ion)
        f_ion = np.empty_like(x_ion)
        self._check(self.lib.tree_gpu_get_state(
            self.h, _dp(x_el), _dp(v_el), _dp(f_el), _dp(x_ion), _dp(v_ion),
            _dp(f_ion)))
        return dict(x_el=x_el, v_el=v_el, f_el=f_el, x_ion=x_ion,
                    v_ion=v_ion, f_ion=f_ion)

    def get_state_ptr(self, x_el, v_el, f_el, x_ion, v_ion, f_ion):
        self._check(self.lib.tree_gpu_get_state(
            self.h, _dp(x_el), _dp(v_el), _dp(f_el), _dp(x_ion), _dp(v_ion),
            _dp(f_ion)))

    def direct(self, targets):
        """FP64 direct sum at the current device positions for global target
        indices; returns (f (nt,3), epot (nt,) = 0.5 sum V)."""
        t = np.ascontiguousarray(np.asarray(targets, dtype=np.int64))
        f = np.empty((len(t), 3))
        e = np.empty(len(t))
        self._check(self.lib.tree_gpu_direct(
            self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(t),
            _dp(f), _dp(e)))
        return f, e

    def tree_dump(self, species: int):
        n = ctypes.c_int64()
        self._check(self.lib.tree_gpu_tree_dump(self.h, species, 0, None, None,
                                                None, None, None, None,
                                                ctypes.byref(n)))
        m = n.value
        centre = np.zeros((m, 3))
        mom = np.zeros((m, 10))
        rcrit = np.zeros(m)
        level = np.zeros(m, np.int32)
        skip = np.zeros(m, np.int64)
        pt = np.zeros(m, np.int64)
        lp = ctypes.POINTER(ctypes.c_int64)
        self._check(self.lib.tree_gpu_tree_dump(
            self.h, species, m, _dp(centre), _dp(mom), _dp(rcrit),
            level.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            skip.ctypes.data_as(lp), pt.ctypes.data_as(lp), ctypes.byref(n)))
        return dict(centre=centre, moments=mom, rcrit=rcrit, level=level,
                    skip=skip, pt=pt)

    def net_dump(self):
        """The combined tree of the mixed path, rebuilt from the current device
        positions with every FP64 record written (pre-order):
        centre (m, 3), moments (m, 38) -- n, Q, D[3], q_ion, S[6] (xx yy zz xy
        yz zx), T[10], H[15], 0 -- first, count, level, parent (m,), and the
        sorted particles (n, 4): x, y, z, 1 for ions."""
        n = ctypes.c_int64()
        self._check(self.lib.tree_gpu_net_dump(self.h, 0, None, None, None, None, None,
                                               None, None, ctypes.byref(n)))
        m = n.value
        centre = np.zeros((m, 3))
        mom = np.zeros((m, 38))
        first = np.zeros(m, np.int64)
        count = np.zeros(m, np.int64)
        level = np.zeros(m, np.int32)
        parent = np.zeros(m, np.int64)
        xs = np.zeros((self.n_el + self.n_ion, 4))
        lp = ctypes.POINTER(ctypes.c_int64)
        self._check(self.lib.tree_gpu_net_dump(
            self.h, m, _dp(centre), _dp(mom), first.ctypes.data_as(lp),
            count.ctypes.data_as(lp), level.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            parent.ctypes.data_as(lp), _dp(xs), ctypes.byref(n)))
        return dict(centre=centre, moments=mom, first=first, count=count, level=level,
                    parent=parent, sorted=xs)

    def set_stream(self, stream_handle: int | None):
        """Enqueue later work on a caller's cudaStream_t (an integer handle,
        e.g. torch.cuda.current_stream().cuda_stream); None restores the
        handle's own stream."""
        self._check(self.lib.tree_gpu_set_stream(self.h, stream_handle or None))

    def set_tuning(self, bucket: int = 8, blocks_per_sm: int = 4, order: int = 3):
        self._check(self.lib.tree_gpu_set_tuning(self.h, bucket, blocks_per_sm, order))

    def set_local_expansion(self, max_ratio: float = 0.08):
        """Accepted cells with (group half-diagonal) / (distance to the cell's
        centroid) <= max_ratio are summed into each target group's local
        expansion instead of being evaluated per target; 0 turns it off."""
        self._check(self.lib.tree_gpu_set_local_expansion(self.h, max_ratio))

    # ---- learned MAC ----
    def mac_collect(self, theta_lo=0.2, theta_hi=0.9, rho_lo=0.05, rho_hi=0.9,
                    max_count=16384, keep=1.0, seed=1, cap=1 << 22):
        n = ctypes.c_int64()
        self._check(self.lib.tree_gpu_mac_collect(self.h, theta_lo, theta_hi,
                                                  rho_lo, rho_hi, max_count, keep,
                                                  seed, cap, ctypes.byref(n)))
        return n.value

    def mac_samples(self):
        n = ctypes.c_int64()
        self._check(self.lib.tree_gpu_mac_samples(self.h, None, None, None, 0, ctypes.byref(n)))
        m = n.value
        f = np.zeros((m, 16), np.float32)
        y = np.zeros(m, np.float32)
        e = np.zeros((m, 2), np.float32)
        if m:
            self._check(self.lib.tree_gpu_mac_samples(self.h, _fp(f), _fp(y), _fp(e), m,
                                                      ctypes.byref(n)))
        return f, y, e

    def mac_clear(self):
        self._check(self.lib.tree_gpu_mac_clear(self.h))

    def mac_train(self, epochs=8, batch=8192, lr=2e-3, tau=0.9, seed=1):
        losses = np.zeros(epochs, np.float32)
        self._check(self.lib.tree_gpu_mac_train(self.h, epochs, batch, lr, tau, seed,
                                                _fp(losses)))
        return losses

    def mac_set_model(self, params, stats):
        p = np.ascontiguousarray(params, np.float32)
        s = np.ascontiguousarray(stats, np.float32)
        assert p.size == MLP_PARAMS and s.size == MLP_STATS
        self._check(self.lib.tree_gpu_mac_set_model(self.h, _fp(p), _fp(s)))

    def mac_get_model(self):
        p = np.zeros(MLP_PARAMS, np.float32)
        s = np.zeros(MLP_STATS, np.float32)
        self._check(self.lib.tree_gpu_mac_get_model(self.h, _fp(p), _fp(s)))
        return p, s

    def mac_config(self, eta=1e-5, rho_lo=0.05, rho_hi=0.9):
        self._check(self.lib.tree_gpu_mac_config(self.h, eta, rho_lo, rho_hi))

    def timings(self) -> Timing:
        t = Timing()
        self._check(self.lib.tree_gpu_timings(self.h, ctypes.byref(t)))
        return t

    def close(self):
        if getattr(self, "h", None):
            self.lib.tree_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Ensemble(TreeForce):
    """Independent clouds of uneven size in one handle: one build, one
    persistent walk launch and one integrator launch per step.  Particles are
    cloud-major (cloud c: n_el[c] electrons, then n_ion[c] ions); every
    TreeForce call that does not depend on the species split (step, run
    without RDF, timings, tuning, learned-MAC model and budget) works."""

    def __init__(self, configs, n_el, n_ion):
        self.lib = load_library()
        self.configs = list(configs)
        self.config = self.configs[0]
        self.n_el_c = np.asarray(n_el, np.int64)
        self.n_ion_c = np.asarray(n_ion, np.int64)
        self.n_el, self.n_ion = int(self.n_el_c.sum()), int(self.n_ion_c.sum())
        self.ncloud = len(self.configs)
        self.offsets = np.concatenate([[0], np.cumsum(self.n_el_c + self.n_ion_c)])
        arr = (Params * self.ncloud)(*[c.to_c() for c in self.configs])
        self._p = arr[0]
        h = ctypes.c_void_p()
        lp = ctypes.POINTER(ctypes.c_int64)
        rc = self.lib.tree_gpu_ensemble_create(arr, self.ncloud,
                                               self.n_el_c.ctypes.data_as(lp),
                                               self.n_ion_c.ctypes.data_as(lp),
                                               ctypes.byref(h))
        if rc != OK:
            raise TreeGpuError(rc, "tree_gpu_ensemble_create failed")
        self.h = h

    @property
    def n(self):
        return self.n_el + self.n_ion

    def set_state(self, x, v):
        self._check(self.lib.tree_gpu_ensemble_set_state(self.h, _dp(x), _dp(v)))

    def load_state(self, x, v, f=None):
        self._check(self.lib.tree_gpu_ensemble_load_state(
            self.h, _dp(x), _dp(v), _dp(f) if f is not None else None))

    def get_state(self):
        x = np.empty((self.n, 3))
        v = np.empty_like(x)
        f = np.empty_like(x)
        self._check(self.lib.tree_gpu_ensemble_get_state(self.h, _dp(x), _dp(v), _dp(f)))
        return dict(x=x, v=v, f=f)

    def get_state_ptr(self, x, v, f):
        """get_state into raw host addresses (pinned buffers)."""
        self._check(self.lib.tree_gpu_ensemble_get_state(self.h, _dp(x), _dp(v), _dp(f)))

    def sums(self):
        """Per-cloud (Epot_e, Epot_i, mv2_el, mv2_ion, rad_el, rad_ion)."""
        out = np.zeros((self.ncloud, 6))
        self._check(self.lib.tree_gpu_ensemble_sums(self.h, _dp(out)))
        return out

    def direct(self, cloud, targets):
        """FP64 direct sum inside one cloud at cloud-local target indices."""
        t = np.ascontiguousarray(targets, np.int64)
        f = np.zeros((len(t), 3))
        e = np.zeros(len(t))
        lp = ctypes.POINTER(ctypes.c_int64)
        self._check(self.lib.tree_gpu_ensemble_direct(self.h, int(cloud), t.ctypes.data_as(lp),
                                                      len(t), _dp(f), _dp(e)))
        return f, e

    def set_config(self, config):
        self.config = config
        self._p = config.to_c()
        self._check(self.lib.tree_gpu_set_params(self.h, ctypes.byref(self._p)))
