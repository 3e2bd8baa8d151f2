"""The host driver on the GPU: a restart-format input run through
tree_b200/tree_run reproduces, in the reference's file formats, what the same
state gives through the library's API (GPU)."""
import os
import subprocess

import numpy as np
import pytest

from tree_b200 import api, build, cloud, units

from test_driver import write_case

pytestmark = pytest.mark.gpu

KB, NREF = 8.617343e-5, 6


def _floats(path):
    rows = [ln.split() for ln in open(path) if ln.strip() and not ln.startswith("#")]
    return np.array([[float(t) for t in r] for r in rows]) if rows else np.zeros((0, 9))


def _xyz(path):
    lines = open(path).read().splitlines()[2:]
    return np.array([[float(t) for t in ln.split()[1:7]] for ln in lines])


def test_driver_matches_the_api(device_lib, tmp_path):
    if not os.path.exists(build.DRIVER):
        build.build_driver()
    c = cloud.make_cloud(2048, seed=77)
    rng = np.random.default_rng(3)
    x = np.vstack([c.x_ion + rng.standard_normal(c.x_ion.shape) * 0.5, c.x_ion])
    v = np.vstack([c.v_el, c.v_ion])
    write_case(tmp_path, x, v)  # tmax 0.2 ns, trest = tdump = 0.1 ns, tsamp 0.05 ns
    r = subprocess.run([build.DRIVER, "--dir", str(tmp_path), "--precision", "fp64"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    names = sorted(os.listdir(tmp_path))
    for f in ("ener000.dat", "ener001.dat", "ener002.dat", "rdf001.dat", "rdf002.dat",
              "res001.xyz", "res002.xyz"):
        assert f in names, names
    # the same state through the API: 21 steps (Nloop_max = 20), samples every 5
    ne = len(x) // 2
    dt = 0.01 / units.TPS
    cfg = api.Config(theta=0.5, rs=0.003, te=50.0, physics=api.PHYS_KELBG,
                     precision=api.PREC_FP64, dx_ei=0.01, dx_ii=0.1)
    with api.TreeForce(ne, ne, cfg) as tf:
        tf.set_state(x[:ne], v[:ne], x[ne:], v[ne:])
        rec1, (ei1, ii1) = tf.run(dt, 10, nsamp=5, rdf=True)
        s10 = tf.get_state()
        rec2, _ = tf.run(dt, 10, nsamp=5, rdf=True)
        s20 = tf.get_state()
    kbm_e = KB * (3 * ne - NREF)
    kbm_i = KB * (3 * ne - NREF)
    e0 = _floats(tmp_path / "ener000.dat")
    e1 = _floats(tmp_path / "ener001.dat")
    assert len(e0) == 2 and len(e1) == 2 and len(_floats(tmp_path / "ener002.dat")) == 0
    for rows, rec in ((e0, rec1), (e1, rec2)):
        t_ns = rec["nloop"] * dt * units.TPS
        te = rec["mv2_el"] / kbm_e
        ti = rec["mv2_ion"] / kbm_i
        epot = rec["epot_e"] + rec["epot_i"]
        etot = 0.5 * (rec["mv2_el"] + rec["mv2_ion"]) + epot
        np.testing.assert_allclose(rows[:, 0], t_ns, rtol=1e-6)
        np.testing.assert_allclose(rows[:, 1], te, rtol=1e-6)
        np.testing.assert_allclose(rows[:, 2], ti, rtol=1e-6)
        np.testing.assert_allclose(rows[:, 7], epot, rtol=1e-6)
        np.testing.assert_allclose(rows[:, 8], etot, rtol=1e-6)
    # restart files: state after steps 10 and 20
    for path, st in (("res001.xyz", s10), ("res002.xyz", s20)):
        r6 = _xyz(tmp_path / path)
        xs = np.vstack([st["x_el"], st["x_ion"]])
        vs = np.vstack([st["v_el"], st["v_ion"]])
        np.testing.assert_allclose(r6[:, :3], xs, rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(r6[:, 3:], vs, rtol=1e-6, atol=1e-12)
    # RDF of the first 10 steps, divided by Ndump (sample.f90:37-39)
    rdf = _floats(tmp_path / "rdf001.dat")
    assert rdf.shape == (api.RDF_BINS, 4)
    np.testing.assert_allclose(rdf[:, 1], ei1 / 10.0, rtol=1e-6)
    np.testing.assert_allclose(rdf[:, 3], ii1 / 10.0, rtol=1e-6)
    assert ei1.sum() > 0
