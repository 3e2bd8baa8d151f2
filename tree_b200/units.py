"""Code units and physical constants of TREE, plus the Kelbg lengths.

Units follow main.f90:188-194 of hpjeonGIT/TREE: length 1 um, mass 1 amu,
energy 1 eV, time 1 tu = 0.10180505305371923 ns (data.f90:39).  In these units
1 amu * (um/tu)^2 = 1 eV, so a = f/m needs no extra factor.
"""
import math

EPS = 0.0014399835661145824       # Coulomb constant, eV*um (data.f90:40)
TPS = 0.10180505305371923         # ns per code time unit (data.f90:39)
KB_EV = 8.617343e-5               # Boltzmann constant, eV/K (main.f90:393)
NREF = 6                          # removed degrees of freedom (data.f90:38)
NDIST = 10000                     # RDF bins = NDIST + 1 (data.f90:38)

M_ELECTRON_AMU = 5.48579909e-4
M_ION_AMU = 88.0

# SI constants for the thermal de Broglie (Kelbg) length.
_HBAR = 1.054571817e-34           # J s
_AMU = 1.66053906660e-27          # kg
_KB_SI = 1.380649e-23             # J/K


def dt_code(dt_seconds: float) -> float:
    """Seconds -> code time units (main.f90:249-254 divides ns by tps)."""
    return dt_seconds * 1e9 / TPS


def kelbg_lambda_um(mu_amu: float, te_kelvin: float) -> float:
    """lambda_ij = hbar / sqrt(2 mu_ij k T_e), in um."""
    return _HBAR / math.sqrt(2.0 * mu_amu * _AMU * _KB_SI * te_kelvin) * 1e6


def kelbg_lambdas(te_kelvin: float, m_e: float = M_ELECTRON_AMU,
                  m_i: float = M_ION_AMU):
    """(lambda_ee, lambda_ei, lambda_ii) in um for reduced masses
    m_e/2, m_e m_i/(m_e+m_i), m_i/2."""
    return (kelbg_lambda_um(m_e / 2.0, te_kelvin),
            kelbg_lambda_um(m_e * m_i / (m_e + m_i), te_kelvin),
            kelbg_lambda_um(m_i / 2.0, te_kelvin))


def sigma_for_density(n_total: int, n0_per_m3: float = 1e15) -> float:
    """Gaussian sigma (um) giving peak density n0 for N particles:
    n0 = N / ((2 pi)^{3/2} sigma^3)."""
    return (n_total / ((2.0 * math.pi) ** 1.5 * n0_per_m3)) ** (1.0 / 3.0) * 1e6
