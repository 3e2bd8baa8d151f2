"""Seeded synthetic ultracold-plasma clouds (the workloads of the benchmarks).

A cloud is an isotropic 3-D Gaussian of ions centred on the origin with every
electron placed at the same point as one ion (t = 0 of an ionised gas).  The
velocities are Maxwellian per component and, like Vinit (main.f90:709-790 of
hpjeonGIT/TREE), rescaled so that sum(m v^2) / (kB (3 N_s - Nref)) equals the
requested temperature exactly for each species.  The reference draws its
velocities from the unseeded Fortran RANDOM_NUMBER; here every draw comes from a
seeded numpy Philox stream so that runs are reproducible.
"""
from dataclasses import dataclass

import numpy as np

from . import units


@dataclass
class Cloud:
    x_el: np.ndarray   # (Ne, 3) float64, um
    v_el: np.ndarray   # (Ne, 3) float64, um/tu
    x_ion: np.ndarray  # (Ni, 3)
    v_ion: np.ndarray
    sigma_um: float

    @property
    def n(self) -> int:
        return len(self.x_el) + len(self.x_ion)


def _maxwell(rng, n, temp_k, mass_amu):
    if n == 0:
        return np.zeros((0, 3))
    v = rng.standard_normal((n, 3)) * np.sqrt(units.KB_EV * temp_k / mass_amu)
    dof = 3 * n - units.NREF
    if dof > 0 and temp_k > 0:
        t0 = float(np.sum(mass_amu * v * v)) / units.KB_EV / dof
        v *= np.sqrt(temp_k / t0)
    return v


def make_cloud(n_total: int, *, seed: int = 1234, te_k: float = 50.0,
               ti_k: float = 1e-3, n0_per_m3: float = 1e15,
               sigma_um: float | None = None,
               m_e: float = units.M_ELECTRON_AMU,
               m_i: float = units.M_ION_AMU,
               colocated: bool = True) -> Cloud:
    """N/2 electrons + N/2 ions.  sigma defaults to the peak-density rule
    sigma = (N / ((2 pi)^{3/2} n0))^{1/3}."""
    if n_total < 0 or n_total % 2:
        raise ValueError("n_total must be a non-negative even number")
    half = n_total // 2
    sig = units.sigma_for_density(n_total, n0_per_m3) if sigma_um is None else sigma_um
    rng = np.random.Generator(np.random.Philox(seed))
    x_ion = rng.standard_normal((half, 3)) * sig
    if colocated:
        x_el = x_ion.copy()
    else:
        x_el = rng.standard_normal((half, 3)) * sig
    v_el = _maxwell(rng, half, te_k, m_e)
    v_ion = _maxwell(rng, half, ti_k, m_i)
    return Cloud(np.ascontiguousarray(x_el), np.ascontiguousarray(v_el),
                 np.ascontiguousarray(x_ion), np.ascontiguousarray(v_ion), sig)
