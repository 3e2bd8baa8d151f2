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


def make_ensemble(ncloud: int = 64, *, seed: int = 5, n_range=(8192, 131072),
                  n0_range=(1e14, 1e16), te_range=(10.0, 200.0), ti_k: float = 1e-3):
    """Independent clouds: N log-uniform in n_range (even), peak density
    log-uniform in n0_range, T_e uniform in te_range; each cloud as
    make_cloud.  Returns (clouds, te per cloud, n0 per cloud)."""
    rng = np.random.Generator(np.random.Philox(seed))
    lo, hi = np.log(n_range[0]), np.log(n_range[1])
    ns = (np.exp(rng.uniform(lo, hi, ncloud)) / 2).astype(np.int64) * 2
    n0 = np.exp(rng.uniform(np.log(n0_range[0]), np.log(n0_range[1]), ncloud))
    te = rng.uniform(te_range[0], te_range[1], ncloud)
    clouds = [make_cloud(int(ns[c]), seed=seed * 1000 + c, te_k=float(te[c]), ti_k=ti_k,
                         n0_per_m3=float(n0[c])) for c in range(ncloud)]
    return clouds, te, n0


def pack_ensemble(clouds):
    """Cloud-major arrays (x, v) and per-cloud (n_el, n_ion) for Ensemble."""
    x = np.vstack([np.vstack([c.x_el, c.x_ion]) for c in clouds])
    v = np.vstack([np.vstack([c.v_el, c.v_ion]) for c in clouds])
    n_el = np.array([len(c.x_el) for c in clouds], np.int64)
    n_ion = np.array([len(c.x_ion) for c in clouds], np.int64)
    return np.ascontiguousarray(x), np.ascontiguousarray(v), n_el, n_ion
