"""The host driver tree_b200/tree_run: reference input formats (CPU, parsing
only via --dry-run; the GPU run is in test_gpu_driver.py)."""
import json
import os
import subprocess

import numpy as np
import pytest

from tree_b200 import build, units

DRIVER = build.DRIVER

CONTROL = """# control file
# charge
-1.0
1.0
# mass (amu)
5.48579909D-4
88.0
# number of electrons, ions
{ne}
{ni}
# temperatures (K)
50.0
0.001
# tmax, trest, tdump, tsamp, dt (ns)
{tmax} {trest}, {tdump}
{tsamp} 0.01
# kelbg, rs
1  0.003
# restart
'{rest}'
# dx_ee, dx_ei, dx_ii
0.01 0.01 0.1
# sd_ratio
0.5
"""


def write_case(d, x, v=None, ids=None, tmax=0.2, trest=0.1, tdump=0.1, tsamp=0.05):
    n = len(x)
    ne = n // 2
    rest = "OFF" if v is None else "ON"
    with open(os.path.join(d, "control.prm"), "w") as f:
        f.write(CONTROL.format(ne=ne, ni=n - ne, tmax=tmax, trest=trest, tdump=tdump,
                               tsamp=tsamp, rest=rest))
    ids = np.arange(1, n + 1) if ids is None else ids
    with open(os.path.join(d, "input.xyz"), "w") as f:
        f.write(f"{n}\nframe = 0\n")
        for i in range(n):
            tag = "P" if i < ne else "O"
            cols = [f"{c:.17g}" for c in x[i]]
            if v is not None:
                cols += [f"{c:.17g}" for c in v[i]]
            f.write(f"{tag} {' '.join(cols)} {ids[i]}\n")


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(DRIVER):
        build.build_driver()
    return DRIVER


def test_dry_run_parses_control_and_positions(driver, tmp_path):
    rng = np.random.default_rng(0)
    x = rng.standard_normal((10, 3)) * 50
    write_case(tmp_path, x)
    out = subprocess.run([driver, "--dir", str(tmp_path), "--dry-run"], capture_output=True,
                         text=True, check=True).stdout
    p = json.loads(out)
    dt = 0.01 / units.TPS
    assert p["nt_el"] == 5 and p["nt_ion"] == 5
    assert p["xm"] == [5.48579909e-4, 88.0]
    assert p["te"] == 50.0 and p["ti"] == 0.001
    assert p["dt"] == pytest.approx(dt, rel=1e-15)
    # Ndump = NINT(tdump/dt) etc. (main.f90:109-116), values across records
    assert (p["ndump"], p["nrest"], p["nsamp"]) == (10, 10, 5)
    # Nloop_max = NINT((tmax + dt/2) / dt) - 1 (main.f90:114-115): NINT of 20.5
    assert p["nloop_max"] == int(np.floor((0.2 / units.TPS + 0.5 * dt) / dt + 0.5)) - 1
    assert p["rs"] == 0.003 and p["rest"] == "OFF" and p["dx"] == [0.01, 0.01, 0.1]
    assert p["sd_ratio"] == 0.5
    assert p["x_first"] == list(x[0]) and p["id_last"] == 10


def test_dry_run_reads_a_restart_file(driver, tmp_path):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((8, 3))
    v = rng.standard_normal((8, 3))
    write_case(tmp_path, x, v, ids=np.arange(100, 108))
    p = json.loads(subprocess.run([driver, "--dir", str(tmp_path), "--dry-run"],
                                  capture_output=True, text=True, check=True).stdout)
    assert p["rest"] == "ON" and p["id_last"] == 107 and p["x_first"] == list(x[0])


def test_missing_inputs_fail_cleanly(driver, tmp_path):
    r = subprocess.run([driver, "--dir", str(tmp_path), "--dry-run"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "control.prm" in r.stderr
