// pair64.cuh -- FP64 leaf pair laws shared by the parity walk and the direct
// sum (both compiled -fmad=false).  Operation order follows tree.f90.
#pragma once
#include "internal.cuh"
#include "walk.h"

namespace tg {

// Adds the force on the target and 0.5*V of one leaf pair.  xr = target -
// source.  Returns false when the pair contributes nothing (REF cutoff of
// same-species pairs, or the target itself in KELBG mode).  `r_out` receives
// the distance for RDF binning when it returns true.
template <int PHYS>
__device__ __forceinline__ bool leaf_pair64(double xr0, double xr1, double xr2,
                                            double r2, bool same, int tsp,
                                            bool is_self, const WalkParams& wp,
                                            double& f0, double& f1, double& f2,
                                            double& ep, double& r_out) {
  if (PHYS == 0) {
    if (same) {
      // Search_Tree_ee/_ii leaf (tree.f90:806-815 / 1115-1131)
      if (!(r2 > 0.01)) return false;
      double r = sqrt(r2);
      const double ff = kEps;
      ep = ep + 0.5 * ff / r;
      f0 = f0 + ff * xr0 / r / r2;
      f1 = f1 + ff * xr1 / r / r2;
      f2 = f2 + ff * xr2 / r / r2;
      r_out = r;
      return true;
    }
    // Search_Tree_ie/_ei leaf (tree.f90:905-913 / 1010-1018); r == 0 gives
    // the r->0 limit instead of the reference's NaN.
    double r = sqrt(r2);
    const double ff = -1.0 * kEps;
    if (r2 == 0.0) {
      ep = ep + 0.5 * ff * (1.0 / wp.rs);
    } else {
      double e = exp(-r / wp.rs);
      ep = ep + 0.5 * ff * (1. - e) / r;
      double g = (1.0 / r - e * (1.0 / r + 1.0 / wp.rs));
      f0 = f0 + ff * xr0 * g / r2;
      f1 = f1 + ff * xr1 * g / r2;
      f2 = f2 + ff * xr2 * g / r2;
    }
    r_out = r;
    return true;
  }
  // erf-Kelbg for every pair (no reference code):
  // V = q q' eps / r [1 - exp(-x^2) + sqrt(pi) x erfc(x)], x = r / lambda
  // F = q q' eps (1 - exp(-x^2)) rhat / r^2
  if (is_self) return false;
  const double qq = same ? 1.0 : -1.0;
  const double lam = same ? (tsp == 0 ? wp.lam_ee : wp.lam_ii) : wp.lam_ei;
  const double pref = qq * kEps;
  const double sqrtpi = 1.7724538509055159;
  if (r2 == 0.0) {
    ep = ep + 0.5 * pref * sqrtpi / lam;
    r_out = 0.0;
    return true;
  }
  double r = sqrt(r2);
  double xx = r / lam;
  double g, ve;
  if (xx * xx > 40.0) {
    // exp(-x^2) < 5e-18 and sqrt(pi) x erfc(x) < 1e-17: both are below half
    // an ulp of 1, so the bracket is 1 to double precision.
    g = 1.0;
    ve = g / r;
  } else {
    g = -expm1(-(xx * xx));
    ve = g / r + sqrtpi * erfc(xx) / lam;
  }
  ep = ep + 0.5 * pref * ve;
  double fr = pref * g / (r2 * r);
  f0 = f0 + fr * xr0;
  f1 = f1 + fr * xr1;
  f2 = f2 + fr * xr2;
  r_out = r;
  return true;
}

}  // namespace tg
