"""C-ABI checks that need no GPU: the library loads, exports every function
include/tree_gpu.h declares, and rejects bad arguments before touching CUDA."""
import ctypes
import os
import re
import subprocess

import pytest

from tree_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tree_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tree_gpu_\w+)\s*\(", text)))


def test_header_lists_the_python_exports():
    assert set(declared_functions()) == set(api.EXPORTS)


def test_library_exports_every_declared_symbol(device_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (tree_gpu_\w+)", out))
    missing = set(declared_functions()) - exported
    assert not missing, f"not exported: {missing}"
    for name in declared_functions():
        assert getattr(device_lib, name) is not None


def test_version_string(device_lib):
    v = device_lib.tree_gpu_version().decode()
    assert "sm_100a" in v


@pytest.mark.parametrize("field,value", [("theta", 0.0), ("theta", float("nan")),
                                         ("physics", 7), ("precision", 9),
                                         ("mac", 5), ("dx_ei", 0.0), ("rs", -1.0)])
def test_create_rejects_bad_params_before_cuda(device_lib, field, value):
    p = api.Config().to_c()
    setattr(p, field, value)
    h = ctypes.c_void_p()
    rc = device_lib.tree_gpu_create(ctypes.byref(p), 4, 4, ctypes.byref(h))
    assert rc == -1 and not h.value


def test_create_rejects_negative_sizes(device_lib):
    p = api.Config().to_c()
    h = ctypes.c_void_p()
    assert device_lib.tree_gpu_create(ctypes.byref(p), -1, 4, ctypes.byref(h)) == -1
    assert device_lib.tree_gpu_create(ctypes.byref(p), 4, 4, None) == -1


def test_null_handle_calls_are_errors(device_lib):
    assert device_lib.tree_gpu_force(None, None, None, None, None, None, None,
                                     None, None) == -1
    assert device_lib.tree_gpu_step(None, 0.1, 1, None) == -1
    assert device_lib.tree_gpu_destroy(None) == 0
    assert b"null" in device_lib.tree_gpu_last_error(None)


def test_fortran_module_declares_every_function():
    """include/tree_gpu_mod.f90 has a BIND(C) interface for each function of
    the header (the module cannot be compiled here: no Fortran compiler)."""
    mod = open(os.path.join(ROOT, "include", "tree_gpu_mod.f90")).read()
    declared = set(re.findall(r"FUNCTION\s+(tree_gpu_\w+)\s*\(", mod))
    assert set(declared_functions()) == declared


def _ensemble_create(lib, cfgs, n_el, n_ion):
    arr = (api.Params * max(1, len(cfgs)))(*[c.to_c() for c in cfgs])
    ne = (ctypes.c_int64 * max(1, len(n_el)))(*n_el)
    ni = (ctypes.c_int64 * max(1, len(n_ion)))(*n_ion)
    h = ctypes.c_void_p()
    rc = lib.tree_gpu_ensemble_create(arr, len(cfgs), ne, ni, ctypes.byref(h))
    return rc, h


def _mixed(**kw):
    return api.Config(precision=api.PREC_MIXED, physics=api.PHYS_KELBG, **kw)


@pytest.mark.parametrize("case", ["no_clouds", "too_many", "fp64_cloud", "mixed_theta",
                                  "negative_size"])
def test_ensemble_create_rejects_bad_arguments_before_cuda(device_lib, case):
    """One walk, one criterion and one integrator serve every cloud, so the
    clouds must agree on precision (mixed), physics, theta, MAC and masses;
    sizes are checked before any device memory is touched."""
    cfgs, ne, ni = [_mixed(te=20.0), _mixed(te=80.0)], [10, 12], [10, 12]
    if case == "no_clouds":
        cfgs, ne, ni = [], [], []
    elif case == "too_many":
        cfgs, ne, ni = [_mixed()] * 257, [2] * 257, [2] * 257
    elif case == "fp64_cloud":
        cfgs[1] = api.Config(precision=api.PREC_FP64, physics=api.PHYS_KELBG)
    elif case == "mixed_theta":
        cfgs[1] = _mixed(theta=0.7)
    elif case == "negative_size":
        ne[1] = -1
    rc, h = _ensemble_create(device_lib, cfgs, ne, ni)
    assert rc == -1 and not h.value


def test_direct_static_checks_arguments_before_cuda(device_lib):
    """The allocation-free audit rejects a target list above its fixed
    scratch size (capacity error) and bad parameters, and returns at once for
    an empty list -- all before any CUDA call."""
    p = _mixed(te=50.0).to_c()
    f = device_lib.tree_gpu_direct_static
    cap = int(re.search(r"#define TREE_GPU_DIRECT_STATIC_MAX_TARGETS (\d+)",
                        open(HEADER).read()).group(1))
    assert f(None, 4, 4, ctypes.byref(p), None, cap + 1, None, None, None) == -4
    assert f(None, 4, 4, ctypes.byref(p), None, -1, None, None, None) == -1
    assert f(None, -4, 4, ctypes.byref(p), None, 1, None, None, None) == -1
    assert f(None, 4, 4, None, None, 1, None, None, None) == -1
    assert f(None, 4, 4, ctypes.byref(p), None, 0, None, None, None) == 0
    bad = _mixed(te=50.0).to_c()
    bad.physics = 7
    assert f(None, 4, 4, ctypes.byref(bad), None, 1, None, None, None) == -1
