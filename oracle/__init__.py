"""ctypes front end of the CPU oracle (liboracle.so, built from tree_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
may import this package.  Parity status: unpinned by the reference (no Fortran
toolchain, no reference fixtures); pinned by the known-answer tests in tests/.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_NATIVE_PATH = os.path.join(_HERE, "liboracle_native.so")
NBINS = 10001

PHYS_REF = 0
PHYS_KELBG = 1


class OracleParams(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_double), ("rs", ctypes.c_double),
                ("dx_ei", ctypes.c_double), ("dx_ii", ctypes.c_double),
                ("lam_ee", ctypes.c_double), ("lam_ei", ctypes.c_double),
                ("lam_ii", ctypes.c_double), ("physics", ctypes.c_int32),
                ("nthreads", ctypes.c_int32)]


class Ref8Stats(ctypes.Structure):
    _fields_ = [("n_el", ctypes.c_int64 * 8), ("n_ion", ctypes.c_int64 * 8),
                ("ghost_nodes_e", ctypes.c_int64), ("ghost_nodes_i", ctypes.c_int64),
                ("n_m2p_ghost", ctypes.c_int64), ("n_p2p_ghost", ctypes.c_int64)]


class OracleStats(ctypes.Structure):
    _fields_ = [("n_m2p", ctypes.c_int64), ("n_p2p", ctypes.c_int64),
                ("max_depth_e", ctypes.c_int32), ("max_depth_i", ctypes.c_int32),
                ("t_build", ctypes.c_double), ("t_walk", ctypes.c_double)]


NODE_DTYPE = np.dtype([("xx", "<f8", 3), ("ox", "<f8", 3), ("lx", "<f8", 3),
                       ("qeff", "<f8"), ("dx", "<f8"), ("D", "<f8", 3),
                       ("Q", "<f8", 3), ("QQ", "<f8", 3), ("pt", "<i8"),
                       ("level", "<i4"), ("ileaf", "<i4"), ("skip", "<i8")])

_lib = None
_flags = "-O3 -march=x86-64-v3 -ffp-contract=off -fopenmp"


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def use_native():
    """Rebuilds the oracle with -march=native on this host (make -B, so a copy
    built on another host is never used) and routes every later call to it.
    Only for the timed CPU baseline; once a library is loaded it stays.
    Returns the compiler flags of the library in use."""
    global _flags
    if _lib is not None:
        return _flags
    try:
        subprocess.run(["make", "-s", "-B", "-C", _HERE, "native"], check=True,
                       capture_output=True, timeout=300)
        _load(_NATIVE_PATH)
        _flags = "-O3 -march=native -ffp-contract=off -fopenmp"
    except (subprocess.SubprocessError, OSError):
        lib()
        _flags += " (native build failed)"
    return _flags


def lib():
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _load(_LIB_PATH)
    return _lib


def _load(path):
    global _lib
    if _lib is None:
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lp = ctypes.POINTER(ctypes.c_int64)
        L.oracle_force.argtypes = [ctypes.c_int64, ctypes.c_int64, dp, dp,
                                   ctypes.POINTER(OracleParams), dp, dp, dp,
                                   lp, lp, ctypes.POINTER(OracleStats)]
        L.oracle_force.restype = ctypes.c_int
        L.oracle_force_strided.argtypes = L.oracle_force.argtypes + [ctypes.c_int64]
        L.oracle_force_strided.restype = ctypes.c_int
        L.oracle_force_ref8.argtypes = L.oracle_force.argtypes + [ctypes.POINTER(Ref8Stats)]
        L.oracle_force_ref8.restype = ctypes.c_int
        L.oracle_tree_dump.argtypes = [ctypes.c_int64, dp, ctypes.c_int32,
                                       ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.POINTER(ctypes.c_int32)]
        L.oracle_tree_dump.restype = ctypes.c_int64
        L.oracle_direct.argtypes = [ctypes.c_int64, ctypes.c_int64, dp, dp,
                                    ctypes.POINTER(OracleParams), lp,
                                    ctypes.c_int64, lp, ctypes.c_int64, dp, dp,
                                    dp]
        L.oracle_direct.restype = ctypes.c_int
        L.oracle_kdk1.argtypes = [ctypes.c_int64, dp, dp, dp, ctypes.c_double,
                                  ctypes.c_double]
        L.oracle_kdk2.argtypes = [ctypes.c_int64, dp, dp, ctypes.c_double,
                                  ctypes.c_double]
        L.oracle_ke.argtypes = [ctypes.c_int64, dp, dp, ctypes.c_double, dp]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _lp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def _c3(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, 3))


def make_params(theta=0.5, rs=0.003, dx_ei=0.01, dx_ii=0.1, lambdas=(1, 1, 1),
                physics=PHYS_REF, nthreads=0):
    return OracleParams(theta, rs, dx_ei, dx_ii, lambdas[0], lambdas[1],
                        lambdas[2], physics, nthreads)


def force(x_el, x_ion, params, rdf=True, stride=1):
    """Tree force (single-domain form of Force, main.f90:506-541).
    stride > 1 walks only every stride-th target (timing samples).

    Returns dict with f_el, f_ion (N,3), epot_e, epot_i, rdf_ei, rdf_ii and
    stats (n_m2p, n_p2p, depths, build/walk seconds)."""
    x_el, x_ion = _c3(x_el), _c3(x_ion)
    f_el = np.zeros_like(x_el)
    f_ion = np.zeros_like(x_ion)
    ep = np.zeros(2)
    rei = np.zeros(NBINS, np.int64)
    rii = np.zeros(NBINS, np.int64)
    st = OracleStats()
    rc = lib().oracle_force_strided(len(x_el), len(x_ion), _dp(x_el),
                                    _dp(x_ion), ctypes.byref(params),
                                    _dp(f_el), _dp(f_ion), _dp(ep),
                                    _lp(rei) if rdf else None,
                                    _lp(rii) if rdf else None,
                                    ctypes.byref(st), int(stride))
    if rc != 0:
        raise RuntimeError(f"oracle_force failed with status {rc}")
    return dict(f_el=f_el, f_ion=f_ion, epot_e=ep[0], epot_i=ep[1],
                rdf_ei=rei, rdf_ii=rii,
                stats=dict(n_m2p=st.n_m2p, n_p2p=st.n_p2p,
                           max_depth_e=st.max_depth_e,
                           max_depth_i=st.max_depth_i,
                           t_build=st.t_build, t_walk=st.t_walk))


def force_ref8(x_el, x_ion, params, rdf=True):
    """Force in the reference's 8-rank form (REF8): one domain per coordinate
    octant, local trees walked locally, pruned ghost trees of the other seven
    ranks walked with their unexpanded twigs as bare monopoles
    (main.f90:506-701, tree.f90:1167-2330).  Same returns as force(), plus
    "ref8": particles per rank, ghost-tree nodes and ghost interactions."""
    x_el, x_ion = _c3(x_el), _c3(x_ion)
    f_el = np.zeros_like(x_el)
    f_ion = np.zeros_like(x_ion)
    ep = np.zeros(2)
    rei = np.zeros(NBINS, np.int64)
    rii = np.zeros(NBINS, np.int64)
    st = OracleStats()
    s8 = Ref8Stats()
    rc = lib().oracle_force_ref8(len(x_el), len(x_ion), _dp(x_el), _dp(x_ion),
                                 ctypes.byref(params), _dp(f_el), _dp(f_ion), _dp(ep),
                                 _lp(rei) if rdf else None, _lp(rii) if rdf else None,
                                 ctypes.byref(st), ctypes.byref(s8))
    if rc != 0:
        raise RuntimeError(f"oracle_force_ref8 failed with status {rc}")
    return dict(f_el=f_el, f_ion=f_ion, epot_e=ep[0], epot_i=ep[1],
                rdf_ei=rei, rdf_ii=rii,
                stats=dict(n_m2p=st.n_m2p, n_p2p=st.n_p2p,
                           max_depth_e=st.max_depth_e, max_depth_i=st.max_depth_i,
                           t_build=st.t_build, t_walk=st.t_walk),
                ref8=dict(n_el=list(s8.n_el), n_ion=list(s8.n_ion),
                          ghost_nodes_e=s8.ghost_nodes_e, ghost_nodes_i=s8.ghost_nodes_i,
                          n_m2p_ghost=s8.n_m2p_ghost, n_p2p_ghost=s8.n_p2p_ghost))


def tree_dump(x, sign):
    """Pre-order node dump of one species tree (sign -1 e, +1 ion)."""
    x = _c3(x)
    cap = max(16, 4 * len(x) + 16)
    while True:
        out = np.zeros(cap, NODE_DTYPE)
        md = ctypes.c_int32(0)
        n = lib().oracle_tree_dump(len(x), _dp(x), sign,
                                   out.ctypes.data_as(ctypes.c_void_p), cap,
                                   ctypes.byref(md))
        if n < 0:
            raise RuntimeError(f"oracle_tree_dump failed with status {n}")
        if n <= cap:
            return out[:n], md.value
        cap = n


def direct(x_el, x_ion, params, t_el=None, t_ion=None):
    """FP64 O(N^2) direct sum on target index lists (default: all)."""
    x_el, x_ion = _c3(x_el), _c3(x_ion)
    t_el = np.arange(len(x_el), dtype=np.int64) if t_el is None else np.ascontiguousarray(t_el, np.int64)
    t_ion = np.arange(len(x_ion), dtype=np.int64) if t_ion is None else np.ascontiguousarray(t_ion, np.int64)
    f_el = np.zeros((len(t_el), 3))
    f_ion = np.zeros((len(t_ion), 3))
    ep = np.zeros(1)
    rc = lib().oracle_direct(len(x_el), len(x_ion), _dp(x_el), _dp(x_ion),
                             ctypes.byref(params), _lp(t_el), len(t_el),
                             _lp(t_ion), len(t_ion), _dp(f_el), _dp(f_ion),
                             _dp(ep))
    if rc != 0:
        raise RuntimeError(f"oracle_direct failed with status {rc}")
    return dict(f_el=f_el, f_ion=f_ion, epot=ep[0])


def kdk1(x, v, f, dt, xm):
    """VVerletNotemp1 in place (vverlet.f90:24-30)."""
    lib().oracle_kdk1(len(x), _dp(x), _dp(v), _dp(f), dt, xm)


def kdk2(v, f, dt, xm):
    """VVerletNotemp2 kick in place (vverlet.f90:64-76)."""
    lib().oracle_kdk2(len(v), _dp(v), _dp(f), dt, xm)


def ke(x, v, xm):
    out = np.zeros(2)
    lib().oracle_ke(len(x), _dp(_c3(x)), _dp(_c3(v)), xm, _dp(out))
    return out[0], out[1]


def max_threads():
    return lib().oracle_max_threads()
