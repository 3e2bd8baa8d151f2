"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference (Fortran90 + MPI) ships no tests, inputs or golden vectors and
cannot be compiled on this image, so these fixtures are produced by the oracle
(oracle/tree_oracle.cpp) after it passes its analytic known-answer tests.  They
pin the oracle against regressions and give the device tests fixed answers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tree_b200 import cloud, units  # noqa: E402


def displaced_cloud(n, seed, shift_um=0.3):
    """Gaussian cloud with each electron displaced from its ion by a seeded
    offset (the state a few steps after t=0, when e-i pairs have separated)."""
    c = cloud.make_cloud(n, seed=seed)
    rng = np.random.Generator(np.random.Philox(seed + 99))
    x_el = c.x_ion + rng.standard_normal(c.x_ion.shape) * shift_um
    return x_el, c.x_ion, c


def case(name, x_el, x_ion, theta, physics, te=50.0):
    lam = units.kelbg_lambdas(te)
    p = oracle.make_params(theta=theta, rs=lam[1], dx_ei=0.01, dx_ii=0.1,
                           lambdas=lam, physics=physics)
    r = oracle.force(x_el, x_ion, p)
    te_dump, _ = oracle.tree_dump(x_el, -1)
    ti_dump, _ = oracle.tree_dump(x_ion, +1)
    return {
        f"{name}_x_el": x_el, f"{name}_x_ion": x_ion,
        f"{name}_theta": np.float64(theta), f"{name}_physics": np.int32(physics),
        f"{name}_te": np.float64(te), f"{name}_rs": np.float64(lam[1]),
        f"{name}_f_el": r["f_el"], f"{name}_f_ion": r["f_ion"],
        f"{name}_epot": np.array([r["epot_e"], r["epot_i"]]),
        f"{name}_rdf_ei": r["rdf_ei"], f"{name}_rdf_ii": r["rdf_ii"],
        f"{name}_tree_e": te_dump, f"{name}_tree_i": ti_dump,
    }


def main():
    out = {}
    xe, xi, _ = displaced_cloud(64, 11)
    out.update(case("small_ref", xe, xi, 0.5, oracle.PHYS_REF))
    out.update(case("small_kelbg", xe, xi, 0.5, oracle.PHYS_KELBG))
    xe, xi, _ = displaced_cloud(1024, 12)
    out.update(case("mid_ref", xe, xi, 0.5, oracle.PHYS_REF))
    c = cloud.make_cloud(512, seed=13)  # co-located t=0 state of config 1
    out.update(case("coloc_ref", c.x_el, c.x_ion, 0.5, oracle.PHYS_REF))
    path = os.path.join(HERE, "golden_forces.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
