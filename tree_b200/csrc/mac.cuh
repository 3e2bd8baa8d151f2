// mac.cuh -- features of a (target group, cell) pair for the learned
// multipole acceptance criterion, shared by the sampling walk (training data)
// and the mixed walk (inference) so both see identical inputs.
//
// All 16 features are dimensionless.  With X the cell centroid, d the
// distance from X to the group's bounding box, u the unit vector from X to
// the group centre, s the cell's box side, dx = |X - geometric centre|, n the
// particle count, Q/D/S/T the net monopole/dipole/second/third moments and
// q_ion the ion count:
//   0 s/d            1 dx/d              2 |h|/d (group half-diagonal)
//   3 log2(n)/16     4 Q/n               5 |D|/(n s)
//   6 |S|_F/(n s^2)  7 log10(|T|_F/(n s^3))/4   8 q_ion/n (species mix)
//   9 D.u/(n s)      10 u.S.u/(n s^2)    11 T(u,u,u)/(n s^3)
//   12 group fill    13 |G-X|/d - 1      14 log10(s/d)
//   15 log10(|T|_F / (n d^3)): the octupole field relative to the gross
//      monopole field n/d^2.
// S and T are the trace-free net moments (|S|_F is stored in geom.w).
// The label is log10(max over the group of |F_multipole - F_exact| /
// (n / d^2)), i.e. the acceptance error relative to the cell's gross
// monopole field (charges in units of e, Coulomb constant dropped).
//
// Pre-filter: before a cell is queued for the network the walk compares a
// log-linear estimate of its label, est = c0 f14 + c1 f3 + c2 f7 + c3 f6 + c4,
// with the budget.  The coefficients are a least-squares fit to the training
// labels and the margins (m_lo, m_hi) are low and high quantiles of
// label - est; both are stored with the model (mlp.cu: mlp_train).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "mlp.cuh"

namespace tg {

constexpr int kMacFeatures = kMlpIn;  // 16

struct CellGeom {   // mx.geom: (s, dx, n, -)
  float s, dx, n, pad;
};

constexpr int kEstCoef = 5;  // pre-filter coefficients (stats[66..70])

__device__ __forceinline__ float mac_estimate(float tnorm, float n, float d) {
  return log10f(tnorm / (n * d * d * d) + 1e-30f);
}

// Features 3, 6, 7 and 14, computed identically for the network and the
// pre-filter.  s, n, |S|_F from geom; tnorm = |T|_F.
__device__ __forceinline__ float mac_f3(float n) { return log2f(n) * (1.f / 16.f); }
__device__ __forceinline__ float mac_f6(float snorm, float n, float s) {
  return snorm / (n * s * s);
}
__device__ __forceinline__ float mac_f7(float tnorm, float n, float s) {
  return log10f(tnorm / (n * s * s * s) + 1e-12f) * 0.25f;
}
__device__ __forceinline__ float mac_f14(float s, float d) { return log10f(s / d); }

// The walk evaluates the estimate split into a part of the cell alone and a
// part of the distance.  With B = log10(budget d^2 / n) the budget in the label's units,
//   est - B = K - log10(budget) - (2 + c0) log10(d),
//   K = c0 log10(s) + c1 f3 + c2 f7 + c3 f6 + c4 + log10(n),
// so K is computed once per cell and build (k_mac_node_terms) and the walk
// compares est + m with B by one logarithm of d.
__device__ __forceinline__ float mac_node_term(const float4 g4, float tnorm, const float* c) {
  const float s = g4.x, n = g4.z;
  return fmaf(c[0], log10f(s),
              fmaf(c[1], mac_f3(n),
                   fmaf(c[2], mac_f7(tnorm, n, s),
                        fmaf(c[3], mac_f6(g4.w, n, s), c[4] + log10f(n)))));
}

__device__ __forceinline__ void mac_features(
    double cx, double cy, double cz, const float4 g4, const float4 m0,
    const float4 m1, const float4 m2, const float4 t0, const float4 t1,
    const float4 t2, double Gx, double Gy, double Gz, float hlen, float d,
    float n_act, float* f) {
  const float s = g4.x, dxo = g4.y, n = g4.z;
  const float Q = m0.x, Dx = m0.y, Dy = m0.z, Dz = m0.w;
  const float Sxx = m1.x, Syy = m1.y, Szz = m1.z, Sxy = m1.w;
  const float Syz = m2.x, Szx = m2.y, qi = m2.w;
  const float ux0 = (float)(Gx - cx), uy0 = (float)(Gy - cy), uz0 = (float)(Gz - cz);
  const float ul = sqrtf(ux0 * ux0 + uy0 * uy0 + uz0 * uz0);
  const float iu = ul > 0.f ? 1.f / ul : 0.f;
  const float ux = ux0 * iu, uy = uy0 * iu, uz = uz0 * iu;
  const float id = 1.f / d;
  const float ns = n * s, ns2 = ns * s, ns3 = ns2 * s;
  const float Dn = sqrtf(Dx * Dx + Dy * Dy + Dz * Dz);
  const float Du = Dx * ux + Dy * uy + Dz * uz;
  const float Sux = Sxx * ux + Sxy * uy + Szx * uz;
  const float Suy = Sxy * ux + Syy * uy + Syz * uz;
  const float Suz = Szx * ux + Syz * uy + Szz * uz;
  const float uSu = ux * Sux + uy * Suy + uz * Suz;
  // T(u,u,u) from the 10 unique components xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
  const float Tuuu = t0.x * ux * ux * ux + t0.y * uy * uy * uy + t0.z * uz * uz * uz +
                     3.f * (t0.w * ux * ux * uy + t1.x * ux * ux * uz + t1.y * ux * uy * uy +
                            t1.z * uy * uy * uz + t1.w * ux * uz * uz + t2.x * uy * uz * uz) +
                     6.f * t2.y * ux * uy * uz;
  const float TF = t2.z;
  f[0] = s * id;
  f[1] = dxo * id;
  f[2] = hlen * id;
  f[3] = mac_f3(n);
  f[4] = Q / n;
  f[5] = Dn / ns;
  f[6] = mac_f6(g4.w, n, s);
  f[7] = mac_f7(TF, n, s);
  f[8] = qi / n;
  f[9] = Du / ns;
  f[10] = uSu / ns2;
  f[11] = Tuuu / ns3;
  f[12] = n_act * (1.f / 32.f);
  f[13] = ul * id - 1.f;
  f[14] = mac_f14(s, d);
  f[15] = mac_estimate(TF, n, d);
}

// Distance from a point to an axis-aligned box (centre G, half extents h).
__device__ __forceinline__ double dist_to_box(double cx, double cy, double cz,
                                              double Gx, double Gy, double Gz,
                                              double hx, double hy, double hz) {
  const double ex = fmax(fabs(cx - Gx) - hx, 0.0);
  const double ey = fmax(fabs(cy - Gy) - hy, 0.0);
  const double ez = fmax(fabs(cz - Gz) - hz, 0.0);
  return sqrt(ex * ex + ey * ey + ez * ez);
}

}  // namespace tg
