"""The allocation-free direct sum (tree_gpu_direct_static) against the
allocating one (tree_gpu_direct), through the C ABI.

tree_gpu_direct_static exists for callers that cannot call cudaMalloc (a host
whose memory manager owns all device memory, or code where an allocation would
synchronise the device or is not allowed); they pass their own device buffers
and the scratch comes from a static device array.  This file is collected last
so that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from tree_b200 import api, cloud

pytestmark = pytest.mark.gpu
TOL = 1e-12  # relative, the direct-sum tolerance of the other GPU tests


def _rel_err(f, g):
    nrm = np.linalg.norm(g, axis=1)
    return np.linalg.norm(f - g, axis=1) / np.maximum(nrm, 1e-3 * nrm.max())


def _static_call(lib, x_dev, n_el, n_ion, params, t_dev, nt, f_dev, e_dev, stream):
    return lib.tree_gpu_direct_static(
        ctypes.c_void_p(x_dev.data_ptr()), n_el, n_ion, ctypes.byref(params),
        ctypes.c_void_p(t_dev.data_ptr()), nt, ctypes.c_void_p(f_dev.data_ptr()),
        ctypes.c_void_p(e_dev.data_ptr()), ctypes.c_void_p(stream))


@pytest.mark.parametrize("physics", [api.PHYS_KELBG, api.PHYS_REF])
def test_static_direct_matches_allocating_direct(device_lib, physics):
    import torch
    c = cloud.make_cloud(30000, seed=77)
    rng = np.random.Generator(np.random.Philox(78))
    x_el = c.x_ion + rng.standard_normal(c.x_ion.shape) * 0.3
    x_ion = c.x_ion
    n_el, n_ion = len(x_el), len(x_ion)
    cfg = api.Config(theta=0.5, physics=physics)
    params = cfg.to_c()
    x_all = np.vstack([x_el, x_ion])
    x_dev = torch.from_numpy(x_all.ravel().copy()).cuda()
    stream = torch.cuda.Stream()
    with api.TreeForce(n_el, n_ion, cfg) as tf:
        tf.force(x_el, x_ion)  # puts the same positions on the device
        # two calls in a row, every buffer made before the first
        calls = []
        for nt in (5000, 1234):
            t = np.sort(rng.choice(n_el + n_ion, nt, replace=False)).astype(np.int64)
            f_ref, e_ref = tf.direct(t)
            calls.append(dict(nt=nt, f_ref=f_ref, e_ref=e_ref,
                              t_dev=torch.from_numpy(t).cuda(),
                              f_dev=torch.full((3 * nt,), float("nan"), dtype=torch.float64,
                                               device="cuda"),
                              e_dev=torch.full((nt,), float("nan"), dtype=torch.float64,
                                               device="cuda")))
        torch.cuda.synchronize()
        free = []
        for k, c in enumerate(calls):
            free.append(torch.cuda.mem_get_info()[0])
            rc = _static_call(device_lib, x_dev, n_el, n_ion, params, c["t_dev"], c["nt"],
                              c["f_dev"], c["e_dev"], stream.cuda_stream)
            assert rc == 0, f"call {k}: status {rc}"
            torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        # the first call may load the module that holds the static array; the
        # second takes no device memory at all
        assert free[2] == free[1], f"free device memory changed by {free[1] - free[2]} bytes"
        for k, c in enumerate(calls):
            f = c["f_dev"].cpu().numpy().reshape(-1, 3)
            e = c["e_dev"].cpu().numpy()
            assert np.all(np.isfinite(f)) and np.all(np.isfinite(e)), f"call {k}"
            assert _rel_err(f, c["f_ref"]).max() <= TOL, f"call {k}"
            np.testing.assert_allclose(e, c["e_ref"], rtol=TOL,
                                       atol=TOL * np.abs(c["e_ref"]).max())


def test_static_direct_rejects_oversize_and_bad_indices(device_lib):
    import torch
    x = np.random.default_rng(1).standard_normal((200, 3)) * 10
    x_dev = torch.from_numpy(x.ravel().copy()).cuda()
    params = api.Config(theta=0.5, physics=api.PHYS_KELBG).to_c()
    big = api_max = 65536 + 1
    t_dev = torch.zeros(big, dtype=torch.int64, device="cuda")
    f_dev = torch.zeros(3 * big, dtype=torch.float64, device="cuda")
    e_dev = torch.zeros(big, dtype=torch.float64, device="cuda")
    rc = _static_call(device_lib, x_dev, 100, 100, params, t_dev, api_max, f_dev, e_dev, 0)
    assert rc == -4  # TREE_GPU_ERR_CAPACITY, nothing launched
    t_bad = torch.tensor([0, 5, 200, -3], dtype=torch.int64, device="cuda")
    rc = _static_call(device_lib, x_dev, 100, 100, params, t_bad, 4, f_dev, e_dev, 0)
    assert rc == -1  # out-of-range indices are reported, never dereferenced
    t_ok = torch.tensor([0, 5, 199], dtype=torch.int64, device="cuda")
    rc = _static_call(device_lib, x_dev, 100, 100, params, t_ok, 3, f_dev, e_dev, 0)
    assert rc == 0  # the error word was cleared for the next call
