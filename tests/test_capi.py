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
