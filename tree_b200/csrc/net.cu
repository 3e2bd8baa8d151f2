// net.cu -- net-charge moments of the combined tree (mixed-precision path).
//
// Compiled with multiply-add contraction on: these moments feed only the
// mixed-precision walk (FP32 far field, FP64 labels of the learned
// criterion), never the FP64 parity path, so their rounding is free.
#include <cstdio>
#include "internal.cuh"
#include "build.h"

namespace tg {

// ------------------------------------------------ net-charge upward pass ----
// multiplicities of the unique index triples of a symmetric 3-tensor, in
// the order xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
__constant__ double kTMult[10] = {1, 1, 1, 3, 3, 3, 3, 3, 3, 6};

// Combined tree (both species in one tree) for the mixed-precision walk.  Per
// twig: particle count n, centroid X (the expansion centre), net charge Q,
// ion count, dipole D = sum q a, second moment S = 1/2 sum q a a^T, third
// moment T_ijk = sum q a_i a_j a_k and fourth moment H_ijkl = sum q a_i a_j
// a_k a_l (a = x - X).  In a quasi-neutral plasma Q ~ 0 for large cells and
// the far field is the small net (dipole, quadrupole, ...) field, so its
// truncation error is relative to that net field rather than to each
// species' monopole.
//
// Twigs of at most kMidCount particles sum their particles directly (P2M):
// every such twig is independent of the others, so the whole lower tree is
// one parallel pass with no waiting on children.  The few twigs above are
// combined from their children by the parallel-axis rules (d_c = X_c - X):
//   D = sum D_c + Q_c d_c,
//   S = sum S_c + (D_c d_c^T + d_c D_c^T)/2 + Q_c d_c d_c^T / 2,
//   T += T_c + d_i S2_jk + d_j S2_ik + d_k S2_ij + d_i d_j D_k + d_i D_j d_k
//        + D_i d_j d_k + Q_c d_i d_j d_k      (S2 = 2 S of the child),
//   H += H_c + 4 sym(d T_c) + 6 sym(d d S2_c) + 4 sym(d d d D_c) + Q_c d d d d
// (sym: the distinct index placements); a leaf child is a point charge.
//
// m64 per twig (19 x double2): (n, Q) | (Dx, Dy) | (Dz, q_ion) | (Sxx, Syy) |
// (Szz, Sxy) | (Syz, Szx) | T in the order xxx yyy zzz xxy xxz xyy yyz xzz
// yzz xyz | H in the order xxxx yyyy zzzz xxxy xxxz xyyy yyyz xzzz yzzz xxyy
// xxzz yyzz xxyz xyyz xyzz, 0 (all raw, for the FP64 labels of the learned
// criterion).  The FP32 copies the walk evaluates are trace-free, which drops
// every trace term from the far-field formula (phi = Q/r + D.d/r^3 +
// 3 d.S'.d/r^5 + 5/2 T'(d,d,d)/r^7 + 35/8 H'(d,d,d,d)/r^9):
// S' = S - tr(S)/3 I and T'_ijk = T_ijk - (d_ij V_k + d_ik V_j + d_jk V_i)/5
// with V_k = T_iik.  mom per twig (3 x float4): (Q, Dx, Dy, Dz),
// (S'xx, S'yy, S'zz, Sxy), (Syz, Szx, trace S, q_ion); mom3 per twig
// (3 x float4): (T'xxx, T'yyy, T'zzz, T'xxy), (T'xxz, T'xyy, T'yyz, T'xzz),
// (T'yzz, Txyz, |T'|_F, 0); mom4 per twig (3 x float4): trace-free H'
// (xxxx, xxxy, xxxz, xxyy), (xxyz, xyyy, xyyz, yyyy), (yyyz, xxzz, xyzz,
// yyzz); geom (s, dx, n, |S'|_F).  Leaves carry no moment records: the walk
// sums them as particles and the parallel-axis pass treats them as point
// charges.
constexpr int kMidCount = 2048;   // twigs up to this size: direct sums (P2M)
constexpr int kSmallCount = 64;   // twigs up to this size: a thread each, else a warp

// ---- the records of one twig ----
// The FP32 records and node_c are always written; the FP64 record m64 only
// where it is read: by the parallel-axis pass (children of the large twigs,
// and the large twigs themselves) and, on request, for every twig (the
// learned criterion's training labels, the debug dump).
// Count, centroid, net charge, ion count, dipole and second moment of twig
// cur: node_c (centroid, critical radius smax / theta + |X - box centre|),
// m64[0..5], mom and geom.  gc: the twig's geometric centre.
__device__ void net_store_low(int cur, double nsum, double X0, double X1, double X2,
                              double Q, double qi, double Dx, double Dy, double Dz,
                              double Sxx, double Syy, double Szz, double Sxy, double Syz,
                              double Szx, double4 gc, double smax0, double theta,
                              const int8_t* __restrict__ node_level, double4* node_c,
                              const MixedNodes& mx, bool rec64) {
  const double a0 = X0 - gc.x, a1 = X1 - gc.y, a2 = X2 - gc.z;
  const double dx = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  const int lev = node_level[cur];
  double smax = smax0;
  for (int l = 0; l < lev; ++l) smax = smax * 0.5;
  node_c[cur] = make_double4(X0, X1, X2, smax / theta + dx);
  if (rec64) {
    double2* m = mx.m64 + kM64 * (int64_t)cur;
    m[0] = make_double2(nsum, Q);
    m[1] = make_double2(Dx, Dy);
    m[2] = make_double2(Dz, qi);
    m[3] = make_double2(Sxx, Syy);
    m[4] = make_double2(Szz, Sxy);
    m[5] = make_double2(Syz, Szx);
  }
  const double trS = Sxx + Syy + Szz;
  const double Sxxt = Sxx - trS / 3.0, Syyt = Syy - trS / 3.0, Szzt = Szz - trS / 3.0;
  const double sn = sqrt(Sxxt * Sxxt + Syyt * Syyt + Szzt * Szzt +
                         2.0 * (Sxy * Sxy + Syz * Syz + Szx * Szx));
  float4* f = mx.mom + 3 * (int64_t)cur;
  f[0] = make_float4((float)Q, (float)Dx, (float)Dy, (float)Dz);
  f[1] = make_float4((float)Sxxt, (float)Syyt, (float)Szzt, (float)Sxy);
  f[2] = make_float4((float)Syz, (float)Szx, (float)trS, (float)qi);
  mx.geom[cur] = make_float4((float)smax, (float)dx, (float)nsum, (float)sn);
}

// Third moment T of twig cur (order xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz):
// m64[6..10] and the trace-free mom3 with its Frobenius norm.
__device__ void net_store_T(int cur, const double (&T)[10], const MixedNodes& mx, bool rec64) {
  if (rec64) {
    double2* m = mx.m64 + kM64 * (int64_t)cur;
#pragma unroll
    for (int u = 0; u < 5; ++u) m[6 + u] = make_double2(T[2 * u], T[2 * u + 1]);
  }
  const double Vx = T[0] + T[5] + T[7], Vy = T[3] + T[1] + T[8], Vz = T[4] + T[6] + T[2];
  double Tt[10];
  Tt[0] = T[0] - 0.6 * Vx;
  Tt[1] = T[1] - 0.6 * Vy;
  Tt[2] = T[2] - 0.6 * Vz;
  Tt[3] = T[3] - 0.2 * Vy;
  Tt[4] = T[4] - 0.2 * Vz;
  Tt[5] = T[5] - 0.2 * Vx;
  Tt[6] = T[6] - 0.2 * Vz;
  Tt[7] = T[7] - 0.2 * Vx;
  Tt[8] = T[8] - 0.2 * Vy;
  Tt[9] = T[9];
  double tn = 0.0;
#pragma unroll
  for (int u = 0; u < 10; ++u) tn += kTMult[u] * Tt[u] * Tt[u];
  float4* f3 = mx.mom3 + 3 * (int64_t)cur;
  f3[0] = make_float4((float)Tt[0], (float)Tt[1], (float)Tt[2], (float)Tt[3]);
  f3[1] = make_float4((float)Tt[4], (float)Tt[5], (float)Tt[6], (float)Tt[7]);
  f3[2] = make_float4((float)Tt[8], (float)Tt[9], (float)sqrt(tn), 0.f);
}

// Fourth moment H of twig cur (order xxxx yyyy zzzz xxxy xxxz xyyy yyyz xzzz
// yzzz xxyy xxzz yyzz xxyz xyyz xyzz): m64[11..18] and the 12 components of
// the trace-free H' = H - sym(delta C)/7 + sym(delta delta) tr C/35 with
// C_kl = H_mmkl that the walk's hexadecapole reads.
__device__ void net_store_H(int cur, const double (&H)[15], const MixedNodes& mx, bool rec64) {
  if (rec64) {
    double2* m = mx.m64 + kM64 * (int64_t)cur;
#pragma unroll
    for (int u = 0; u < 7; ++u) m[11 + u] = make_double2(H[2 * u], H[2 * u + 1]);
    m[18] = make_double2(H[14], 0.0);
  }
  const double Cxx = H[0] + H[9] + H[10], Cyy = H[9] + H[1] + H[11],
               Czz = H[10] + H[11] + H[2], Cxy = H[3] + H[5] + H[14],
               Cxz = H[4] + H[13] + H[7], Cyz = H[12] + H[6] + H[8];
  const double c = Cxx + Cyy + Czz;
  const double a7 = 1.0 / 7.0, a35 = 1.0 / 35.0;
  float4* f4 = mx.mom4 + 3 * (int64_t)cur;
  f4[0] = make_float4((float)(H[0] - 6.0 * a7 * Cxx + 3.0 * a35 * c),  // xxxx
                      (float)(H[3] - 3.0 * a7 * Cxy),                  // xxxy
                      (float)(H[4] - 3.0 * a7 * Cxz),                  // xxxz
                      (float)(H[9] - a7 * (Cxx + Cyy) + a35 * c));      // xxyy
  f4[1] = make_float4((float)(H[12] - a7 * Cyz),                       // xxyz
                      (float)(H[5] - 3.0 * a7 * Cxy),                  // xyyy
                      (float)(H[13] - a7 * Cxz),                       // xyyz
                      (float)(H[1] - 6.0 * a7 * Cyy + 3.0 * a35 * c));  // yyyy
  f4[2] = make_float4((float)(H[6] - 3.0 * a7 * Cyz),                  // yyyz
                      (float)(H[10] - a7 * (Cxx + Czz) + a35 * c),     // xxzz
                      (float)(H[14] - a7 * Cxy),                       // xyzz
                      (float)(H[11] - a7 * (Cyy + Czz) + a35 * c));     // yyzz
}

// ---- direct moments (P2M) ----
// Sum over the G lanes of an aligned lane group (butterfly: every lane of the
// group ends with the same total, added in the same order).
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned mask = 0xffffffffu) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

// One sorted particle relative to the centroid: a = x - X, q = +1 ion / -1
// electron, w = 1 ion / 0 electron.
struct P2mPt {
  double ax, ay, az, q, w;
};
__device__ __forceinline__ P2mPt p2m_pt(const double4* __restrict__ xs, int j, double X0,
                                        double X1, double X2) {
  const double4 p = ldg_d4(&xs[j]);
  return {p.x - X0, p.y - X1, p.z - X2, p.w > 0.5 ? 1.0 : -1.0, p.w};
}

// Moments of twig t straight from its particles (the sorted range first ..
// first + count - 1 of xs), one pass per moment order so that few
// accumulators are live: the centroid; Q, q_ion, D and S about it; T; H.
// G lanes share the twig: lane `sub` takes every G-th particle and the group
// adds the lanes' sums after each pass; lane 0 of the group stores.  Every
// lane of the warp calls this together (t < 0: a group without a twig, which
// still takes part in the shuffles).
template <int G>
__device__ void net_p2m(int t, int sub, const Geom* __restrict__ geom, double theta,
                        double4* node_c, const int8_t* __restrict__ node_level,
                        const int32_t* __restrict__ node_parent, const MixedNodes& mx,
                        const Ensemble& ens, bool full) {
  int first = 0, cnt = 0;
  if (t >= 0) {
    first = __ldg(&mx.first[t]);
    cnt = __ldg(&mx.count[t]);
  }
  const double4* __restrict__ xs = mx.xs + first;
  const bool store = t >= 0 && sub == 0;
  // pass 1: centroid
  double X0 = 0.0, X1 = 0.0, X2 = 0.0;
  for (int j = sub; j < cnt; j += G) {
    const double4 p = ldg_d4(&xs[j]);
    X0 += p.x;
    X1 += p.y;
    X2 += p.z;
  }
  X0 = group_sum<G>(X0);
  X1 = group_sum<G>(X1);
  X2 = group_sum<G>(X2);
  const double nsum = (double)cnt;
  if (cnt > 0) {
    X0 /= nsum;
    X1 /= nsum;
    X2 /= nsum;
  }
  bool rec64 = full;
  if (store && !rec64) {
    const int par = __ldg(&node_parent[t]);
    rec64 = par >= 0 && __ldg(&mx.count[par]) > kMidCount;
  }
  // pass 2: Q, q_ion, D and S = 1/2 sum q a a^T
  {
    double Q = 0, qi = 0, Dx = 0, Dy = 0, Dz = 0;
    double Sxx = 0, Syy = 0, Szz = 0, Sxy = 0, Syz = 0, Szx = 0;
    for (int j = sub; j < cnt; j += G) {
      const P2mPt a = p2m_pt(xs, j, X0, X1, X2);
      const double qx = a.q * a.ax, qy = a.q * a.ay, qz = a.q * a.az;
      Q += a.q;
      qi += a.w;
      Dx += qx;
      Dy += qy;
      Dz += qz;
      Sxx += qx * a.ax;
      Syy += qy * a.ay;
      Szz += qz * a.az;
      Sxy += qx * a.ay;
      Syz += qy * a.az;
      Szx += qz * a.ax;
    }
    Q = group_sum<G>(Q);
    qi = group_sum<G>(qi);
    Dx = group_sum<G>(Dx);
    Dy = group_sum<G>(Dy);
    Dz = group_sum<G>(Dz);
    Sxx = 0.5 * group_sum<G>(Sxx);
    Syy = 0.5 * group_sum<G>(Syy);
    Szz = 0.5 * group_sum<G>(Szz);
    Sxy = 0.5 * group_sum<G>(Sxy);
    Syz = 0.5 * group_sum<G>(Syz);
    Szx = 0.5 * group_sum<G>(Szx);
    if (store) {
      const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, first) : 0;
      const double4 gc = ldg_d4(&node_c[t]);  // geometric centre (topology)
      net_store_low(t, nsum, X0, X1, X2, Q, qi, Dx, Dy, Dz, Sxx, Syy, Szz, Sxy, Syz, Szx,
                    gc, geom[seg].smax0, theta, node_level, node_c, mx, rec64);
    }
  }
  // pass 3: T (order xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz)
  {
    double T[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = sub; j < cnt; j += G) {
      const P2mPt a = p2m_pt(xs, j, X0, X1, X2);
      const double qxx = a.q * a.ax * a.ax, qyy = a.q * a.ay * a.ay, qzz = a.q * a.az * a.az;
      T[0] += qxx * a.ax;
      T[1] += qyy * a.ay;
      T[2] += qzz * a.az;
      T[3] += qxx * a.ay;
      T[4] += qxx * a.az;
      T[5] += qyy * a.ax;
      T[6] += qyy * a.az;
      T[7] += qzz * a.ax;
      T[8] += qzz * a.ay;
      T[9] += a.q * a.ax * a.ay * a.az;
    }
#pragma unroll
    for (int u = 0; u < 10; ++u) T[u] = group_sum<G>(T[u]);
    if (store) net_store_T(t, T, mx, rec64);
  }
  // pass 4: H (order xxxx yyyy zzzz xxxy xxxz xyyy yyyz xzzz yzzz xxyy xxzz
  // yyzz xxyz xyyz xyzz)
  {
    double H[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = sub; j < cnt; j += G) {
      const P2mPt a = p2m_pt(xs, j, X0, X1, X2);
      const double qxx = a.q * a.ax * a.ax, qyy = a.q * a.ay * a.ay, qzz = a.q * a.az * a.az;
      H[0] += qxx * a.ax * a.ax;
      H[1] += qyy * a.ay * a.ay;
      H[2] += qzz * a.az * a.az;
      H[3] += qxx * a.ax * a.ay;
      H[4] += qxx * a.ax * a.az;
      H[5] += qyy * a.ay * a.ax;
      H[6] += qyy * a.ay * a.az;
      H[7] += qzz * a.az * a.ax;
      H[8] += qzz * a.az * a.ay;
      H[9] += qxx * a.ay * a.ay;
      H[10] += qxx * a.az * a.az;
      H[11] += qyy * a.az * a.az;
      H[12] += qxx * a.ay * a.az;
      H[13] += qyy * a.ax * a.az;
      H[14] += qzz * a.ax * a.ay;
    }
#pragma unroll
    for (int u = 0; u < 15; ++u) H[u] = group_sum<G>(H[u]);
    if (store) net_store_H(t, H, mx, rec64);
  }
}

// ---- parallel-axis moments of the twigs above ----
// The first K double2 of child c's moment record, or a point charge's (n = 1,
// charge q, ion count) for a leaf.
template <int K>
__device__ __forceinline__ void child_rec(int c, bool leaf, const MixedNodes& mx,
                                          double2 (&r)[K]) {
  if (leaf) {
    const double w = __ldg(&mx.xs[__ldg(&mx.first[c])].w);
#pragma unroll
    for (int u = 0; u < K; ++u) r[u] = make_double2(0.0, 0.0);
    r[0] = make_double2(1.0, w > 0.5 ? 1.0 : -1.0);
    if (K > 2) r[2 % K].y = w;
  } else {
    const double2* cm = mx.m64 + kM64 * (int64_t)c;
#pragma unroll
    for (int u = 0; u < K; ++u) r[u] = __ldcg(cm + u);
  }
}

// Net moments of twig `cur` from its children (all final) by the 8 lanes of
// an aligned lane group (mask gm), lane j taking the child of octant digit j:
// the centroid, then each child's Q, D, S, T and H translated to it by the
// parallel-axis rules and summed over the group (butterfly); lane 0 stores.
// All 8 lanes call this together.
__device__ bool net_twig8(int cur, int j, unsigned gm, double smax0, double theta, int cap,
                          double4* node_c, const int8_t* __restrict__ node_level,
                          const MixedNodes& mx, int32_t* err) {
  const double4 gc = ldcg_d4(&node_c[cur]);  // geometric centre (topology)
  const int c = __ldg(&mx.kids[8 * (int64_t)cur + j]);
  if (__any_sync(gm, c >= cap || (c >= 0 && c <= cur))) {
    if (j == 0) set_error(err, kErrWalk);
    return false;
  }
  double4 cc = make_double4(0.0, 0.0, 0.0, 0.0);
  double2 r[19];
#pragma unroll
  for (int u = 0; u < 19; ++u) r[u] = make_double2(0.0, 0.0);
  if (c >= 0) {
    cc = ldcg_d4(&node_c[c]);
    child_rec<19>(c, cc.w < 0.0, mx, r);
  }
  // centroid: count-weighted child centroids
  const double nc = r[0].x;
  const double nsum = group_sum<8>(nc, gm);
  const double X0 = group_sum<8>(nc * cc.x, gm) / nsum;
  const double X1 = group_sum<8>(nc * cc.y, gm) / nsum;
  const double X2 = group_sum<8>(nc * cc.z, gm) / nsum;
  // this lane's child about the centroid (all zero for an empty octant)
  const double qc = r[0].y, dcx = r[1].x, dcy = r[1].y, dcz = r[2].x;
  const double ex = cc.x - X0, ey = cc.y - X1, ez = cc.z - X2;
  {
    const double Q = group_sum<8>(qc, gm), qi = group_sum<8>(r[2].y, gm);
    const double Dx = group_sum<8>(dcx + qc * ex, gm);
    const double Dy = group_sum<8>(dcy + qc * ey, gm);
    const double Dz = group_sum<8>(dcz + qc * ez, gm);
    const double Sxx = group_sum<8>(r[3].x + dcx * ex + 0.5 * qc * ex * ex, gm);
    const double Syy = group_sum<8>(r[3].y + dcy * ey + 0.5 * qc * ey * ey, gm);
    const double Szz = group_sum<8>(r[4].x + dcz * ez + 0.5 * qc * ez * ez, gm);
    const double Sxy = group_sum<8>(r[4].y + 0.5 * (dcx * ey + ex * dcy) + 0.5 * qc * ex * ey, gm);
    const double Syz = group_sum<8>(r[5].x + 0.5 * (dcy * ez + ey * dcz) + 0.5 * qc * ey * ez, gm);
    const double Szx = group_sum<8>(r[5].y + 0.5 * (dcz * ex + ez * dcx) + 0.5 * qc * ez * ex, gm);
    if (j == 0)
      net_store_low(cur, nsum, X0, X1, X2, Q, qi, Dx, Dy, Dz, Sxx, Syy, Szz, Sxy, Syz, Szx,
                    gc, smax0, theta, node_level, node_c, mx, true);
  }
  const double S2xx = 2 * r[3].x, S2yy = 2 * r[3].y, S2zz = 2 * r[4].x, S2xy = 2 * r[4].y,
               S2yz = 2 * r[5].x, S2xz = 2 * r[5].y;
  {
    double Tc[10], T[10];
#pragma unroll
    for (int u = 0; u < 5; ++u) {
      Tc[2 * u] = r[6 + u].x;
      Tc[2 * u + 1] = r[6 + u].y;
    }
#pragma unroll
    for (int u = 0; u < 10; ++u) T[u] = 0.0;
    T[0] += Tc[0] + ex * S2xx + ex * S2xx + ex * S2xx + ex * ex * dcx + ex * dcx * ex + dcx * ex * ex + qc * ex * ex * ex;
    T[1] += Tc[1] + ey * S2yy + ey * S2yy + ey * S2yy + ey * ey * dcy + ey * dcy * ey + dcy * ey * ey + qc * ey * ey * ey;
    T[2] += Tc[2] + ez * S2zz + ez * S2zz + ez * S2zz + ez * ez * dcz + ez * dcz * ez + dcz * ez * ez + qc * ez * ez * ez;
    T[3] += Tc[3] + ex * S2xy + ex * S2xy + ey * S2xx + ex * ex * dcy + ex * dcx * ey + dcx * ex * ey + qc * ex * ex * ey;
    T[4] += Tc[4] + ex * S2xz + ex * S2xz + ez * S2xx + ex * ex * dcz + ex * dcx * ez + dcx * ex * ez + qc * ex * ex * ez;
    T[5] += Tc[5] + ex * S2yy + ey * S2xy + ey * S2xy + ex * ey * dcy + ex * dcy * ey + dcx * ey * ey + qc * ex * ey * ey;
    T[6] += Tc[6] + ey * S2yz + ey * S2yz + ez * S2yy + ey * ey * dcz + ey * dcy * ez + dcy * ey * ez + qc * ey * ey * ez;
    T[7] += Tc[7] + ex * S2zz + ez * S2xz + ez * S2xz + ex * ez * dcz + ex * dcz * ez + dcx * ez * ez + qc * ex * ez * ez;
    T[8] += Tc[8] + ey * S2zz + ez * S2yz + ez * S2yz + ey * ez * dcz + ey * dcz * ez + dcy * ez * ez + qc * ey * ez * ez;
    T[9] += Tc[9] + ex * S2yz + ey * S2xz + ez * S2xy + ex * ey * dcz + ex * dcy * ez + dcx * ey * ez + qc * ex * ey * ez;
#pragma unroll
    for (int u = 0; u < 10; ++u) T[u] = group_sum<8>(T[u], gm);
    if (j == 0) net_store_T(cur, T, mx, true);
  }
  {
    const double Txxx = r[6].x, Tyyy = r[6].y, Tzzz = r[7].x, Txxy = r[7].y, Txxz = r[8].x,
                 Txyy = r[8].y, Tyyz = r[9].x, Txzz = r[9].y, Tyzz = r[10].x, Txyz = r[10].y;
    double Hc[16], H[15];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      Hc[2 * u] = r[11 + u].x;
      Hc[2 * u + 1] = r[11 + u].y;
    }
#pragma unroll
    for (int u = 0; u < 15; ++u) H[u] = 0.0;
    H[0] += Hc[0] + 4.0 * ex * Txxx + 6.0 * ex * ex * S2xx + 4.0 * ex * ex * ex * dcx + qc * ex * ex * ex * ex;
    H[1] += Hc[1] + 4.0 * ey * Tyyy + 6.0 * ey * ey * S2yy + 4.0 * ey * ey * ey * dcy + qc * ey * ey * ey * ey;
    H[2] += Hc[2] + 4.0 * ez * Tzzz + 6.0 * ez * ez * S2zz + 4.0 * ez * ez * ez * dcz + qc * ez * ez * ez * ez;
    H[3] += Hc[3] + 3.0 * ex * Txxy + ey * Txxx + 3.0 * ex * ex * S2xy + 3.0 * ex * ey * S2xx + 3.0 * ex * ex * ey * dcx + ex * ex * ex * dcy + qc * ex * ex * ex * ey;
    H[4] += Hc[4] + 3.0 * ex * Txxz + ez * Txxx + 3.0 * ex * ex * S2xz + 3.0 * ex * ez * S2xx + 3.0 * ex * ex * ez * dcx + ex * ex * ex * dcz + qc * ex * ex * ex * ez;
    H[5] += Hc[5] + ex * Tyyy + 3.0 * ey * Txyy + 3.0 * ex * ey * S2yy + 3.0 * ey * ey * S2xy + ey * ey * ey * dcx + 3.0 * ex * ey * ey * dcy + qc * ex * ey * ey * ey;
    H[6] += Hc[6] + 3.0 * ey * Tyyz + ez * Tyyy + 3.0 * ey * ey * S2yz + 3.0 * ey * ez * S2yy + 3.0 * ey * ey * ez * dcy + ey * ey * ey * dcz + qc * ey * ey * ey * ez;
    H[7] += Hc[7] + ex * Tzzz + 3.0 * ez * Txzz + 3.0 * ex * ez * S2zz + 3.0 * ez * ez * S2xz + ez * ez * ez * dcx + 3.0 * ex * ez * ez * dcz + qc * ex * ez * ez * ez;
    H[8] += Hc[8] + ey * Tzzz + 3.0 * ez * Tyzz + 3.0 * ey * ez * S2zz + 3.0 * ez * ez * S2yz + ez * ez * ez * dcy + 3.0 * ey * ez * ez * dcz + qc * ey * ez * ez * ez;
    H[9] += Hc[9] + 2.0 * ex * Txyy + 2.0 * ey * Txxy + ex * ex * S2yy + 4.0 * ex * ey * S2xy + ey * ey * S2xx + 2.0 * ex * ey * ey * dcx + 2.0 * ex * ex * ey * dcy + qc * ex * ex * ey * ey;
    H[10] += Hc[10] + 2.0 * ex * Txzz + 2.0 * ez * Txxz + ex * ex * S2zz + 4.0 * ex * ez * S2xz + ez * ez * S2xx + 2.0 * ex * ez * ez * dcx + 2.0 * ex * ex * ez * dcz + qc * ex * ex * ez * ez;
    H[11] += Hc[11] + 2.0 * ey * Tyzz + 2.0 * ez * Tyyz + ey * ey * S2zz + 4.0 * ey * ez * S2yz + ez * ez * S2yy + 2.0 * ey * ez * ez * dcy + 2.0 * ey * ey * ez * dcz + qc * ey * ey * ez * ez;
    H[12] += Hc[12] + 2.0 * ex * Txyz + ey * Txxz + ez * Txxy + ex * ex * S2yz + 2.0 * ex * ey * S2xz + 2.0 * ex * ez * S2xy + ey * ez * S2xx + 2.0 * ex * ey * ez * dcx + ex * ex * ez * dcy + ex * ex * ey * dcz + qc * ex * ex * ey * ez;
    H[13] += Hc[13] + ex * Tyyz + 2.0 * ey * Txyz + ez * Txyy + 2.0 * ex * ey * S2yz + ex * ez * S2yy + ey * ey * S2xz + 2.0 * ey * ez * S2xy + ey * ey * ez * dcx + 2.0 * ex * ey * ez * dcy + ex * ey * ey * dcz + qc * ex * ey * ey * ez;
    H[14] += Hc[14] + ex * Tyzz + ey * Txzz + 2.0 * ez * Txyz + ex * ey * S2zz + 2.0 * ex * ez * S2yz + 2.0 * ey * ez * S2xz + ez * ez * S2xy + ey * ez * ez * dcx + ex * ez * ez * dcy + 2.0 * ex * ey * ez * dcz + qc * ex * ey * ez * ez;
#pragma unroll
    for (int u = 0; u < 15; ++u) H[u] = group_sum<8>(H[u], gm);
    if (j == 0) net_store_H(cur, H, mx, true);
  }
  return true;
}

// ---- the pass ----
// Twigs are sorted into work classes by particle count: 32-64, 16-31, 8-15,
// 4-7 and 2-3 (one thread each, in that order, so that a warp's twigs take
// about as many iterations), 65 .. kMidCount (a warp each), and the twigs
// above kMidCount whose twig children are all below it (where the
// parallel-axis climb starts).  The other twigs above kMidCount count the
// children of their own kind that they wait for in node_done.  The sort is a
// counting sort over blocks of kNetBlockNodes nodes: per-block class counts
// (class-major), their exclusive scan, then each block writes its twigs of
// each class in index order at its offset -- the list holds the classes in
// order and every class in node order.
constexpr int kNetClasses = 7;  // class index: 0..4 one thread, 5 a warp, 6 climb start
constexpr int kNetThreads = 256;
constexpr int kNetNodesPerThread = 4;
constexpr int kNetBlockNodes = kNetThreads * kNetNodesPerThread;
static_assert(kNetBlockNodes == 1024, "net_cls_entries assumes blocks of 1024 nodes");

__device__ __forceinline__ int net_class_of(int c) {
  if (c > kMidCount) return 6;
  if (c > kSmallCount) return 5;
  return c >= 32 ? 0 : c >= 16 ? 1 : c >= 8 ? 2 : c >= 4 ? 3 : 4;
}

// Class of twig i (-1: a leaf, or a large twig reached by the climb); sets
// node_done of the large twigs when `mark` is on.
__device__ __forceinline__ int net_class(int i, int cap, const int32_t* __restrict__ node_pt,
                                         const MixedNodes& mx, int32_t* node_done,
                                         bool mark) {
  if (node_pt[i] >= 0) return -1;
  const int k = net_class_of(mx.count[i]);
  if (k != 6) return k;
  if (!mark) return node_done[i] == 0 ? 6 : -1;
  const int4* kk = reinterpret_cast<const int4*>(mx.kids + 8 * (int64_t)i);
  const int4 k0 = kk[0], k1 = kk[1];
  const int kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
  int big = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j)
    big += (kv[j] >= 0 && kv[j] < cap && node_pt[kv[j]] < 0 && mx.count[kv[j]] > kMidCount)
               ? 1 : 0;
  node_done[i] = big;
  return big == 0 ? 6 : -1;
}

// Pass 1 of the sort: class counts of node block b (nodes b kNetBlockNodes
// .. + kNetBlockNodes - 1) in cnt[class * NB + b], for the blocks that hold
// nodes (the grid strides over them; NB: the blocks of the node capacity).
__global__ void __launch_bounds__(kNetThreads)
    k_net_mark(const int32_t* __restrict__ bounds, int cap, int NB,
               const int32_t* __restrict__ node_pt, int32_t* node_done, MixedNodes mx,
               int32_t* cnt) {
  __shared__ int32_t h[kNetClasses];
  const int m = bounds[2] < cap ? bounds[2] : cap;
  const int nblk = (m + kNetBlockNodes - 1) / kNetBlockNodes;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    if (threadIdx.x < kNetClasses) h[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kNetNodesPerThread; ++u) {
      const int i = blk * kNetBlockNodes + u * kNetThreads + threadIdx.x;
      if (i < m) {
        const int k = net_class(i, cap, node_pt, mx, node_done, true);
        if (k >= 0) atomicAdd(&h[k], 1);
      }
    }
    __syncthreads();
    if (threadIdx.x < kNetClasses) cnt[threadIdx.x * NB + blk] = h[threadIdx.x];
    __syncthreads();
  }
}

// The exclusive scan of the counts in class-major order, one block: off[c *
// NB + b] = where block b's twigs of class c start; start[c] = where class c
// starts (start[7] = all twigs listed).
__global__ void __launch_bounds__(1024)
    k_net_scan(const int32_t* __restrict__ bounds, int cap, int NB,
               const int32_t* __restrict__ cnt, int32_t* off, int32_t* start) {
  __shared__ int32_t ws[32];
  __shared__ int32_t carry;
  const int m = bounds[2] < cap ? bounds[2] : cap;
  const int nblk = (m + kNetBlockNodes - 1) / kNetBlockNodes;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int c = 0; c < kNetClasses; ++c) {
    if (threadIdx.x == 0) start[c] = carry;
    for (int b0 = 0; b0 < nblk; b0 += 1024) {
      const int b = b0 + threadIdx.x;
      const int v = b < nblk ? cnt[c * NB + b] : 0;
      int inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane == 31) ws[w] = inc;
      __syncthreads();
      if (w == 0) {
        const int x = ws[lane];
        int wi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, wi, o);
          if (lane >= o) wi += t;
        }
        ws[lane] = wi - x;
      }
      __syncthreads();
      const int base = carry;
      if (b < nblk) off[c * NB + b] = base + ws[w] + inc - v;
      __syncthreads();
      if (threadIdx.x == 1023) carry = base + ws[w] + inc;
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) start[kNetClasses] = carry;
}

// Pass 2: block b's twigs of class c written in index order from off[c * NB
// + b].
__global__ void __launch_bounds__(kNetThreads)
    k_net_fill(const int32_t* __restrict__ bounds, int cap, int NB,
               const int32_t* __restrict__ node_pt, int32_t* node_done, MixedNodes mx,
               const int32_t* __restrict__ off, int32_t* list) {
  __shared__ int32_t s_w[kNetClasses][kNetThreads / 32];  // per-warp starts
  __shared__ int32_t s_run[kNetClasses];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int m = bounds[2] < cap ? bounds[2] : cap;
  const int nblk = (m + kNetBlockNodes - 1) / kNetBlockNodes;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    if (threadIdx.x < kNetClasses) s_run[threadIdx.x] = off[threadIdx.x * NB + blk];
    __syncthreads();
    for (int u = 0; u < kNetNodesPerThread; ++u) {
      const int i = blk * kNetBlockNodes + u * kNetThreads + threadIdx.x;
      const int k = i < m ? net_class(i, cap, node_pt, mx, node_done, false) : -1;
      int rank = 0;
#pragma unroll
      for (int c = 0; c < kNetClasses; ++c) {
        const unsigned bm = __ballot_sync(0xffffffffu, k == c);
        if (k == c) rank = __popc(bm & lt);
        if (lane == 0) s_w[c][w] = __popc(bm);
      }
      __syncthreads();
      if (threadIdx.x < kNetClasses) {
        int run = s_run[threadIdx.x];
#pragma unroll
        for (int ww = 0; ww < kNetThreads / 32; ++ww) {
          const int t = s_w[threadIdx.x][ww];
          s_w[threadIdx.x][ww] = run;
          run += t;
        }
        s_run[threadIdx.x] = run;
      }
      __syncthreads();
      if (k >= 0) list[s_w[k][w] + rank] = i;
      __syncthreads();
    }
  }
}

// One thread per twig of classes 0..4: list[start[0] .. start[5]).
__global__ void __launch_bounds__(kNetThreads, 4)
    k_net_p2m_thread(const Geom* __restrict__ geom, double theta, double4* node_c,
                     const int8_t* __restrict__ node_level,
                     const int32_t* __restrict__ node_parent, MixedNodes mx, Ensemble ens,
                     const int32_t* __restrict__ start,
                     const int32_t* __restrict__ list, int full, int32_t* err) {
  const int b0 = start[0], b1 = start[5];
  if (*((volatile int32_t*)err) & (kErrCapacity | kErrWalk)) return;
  for (int k = b0 + blockIdx.x * blockDim.x + threadIdx.x; k < b1; k += gridDim.x * blockDim.x)
    net_p2m<1>(list[k], 0, geom, theta, node_c, node_level, node_parent, mx, ens, full != 0);
}

// One warp per twig of class 5: list[start[5] .. start[6]).
__global__ void __launch_bounds__(kNetThreads)
    k_net_p2m_warp(const Geom* __restrict__ geom, double theta, double4* node_c,
                   const int8_t* __restrict__ node_level,
                   const int32_t* __restrict__ node_parent, MixedNodes mx, Ensemble ens,
                   const int32_t* __restrict__ start,
                   const int32_t* __restrict__ list, int full, int32_t* err) {
  const int b0 = start[5], b1 = start[6];
  const int lane = threadIdx.x & 31;
  int e = 0;
  if (lane == 0) e = *((volatile int32_t*)err);
  if (__shfl_sync(0xffffffffu, e, 0) & (kErrCapacity | kErrWalk)) return;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = b0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < b1; k += nw) {
    net_p2m<32>(list[k], lane, geom, theta, node_c, node_level, node_parent, mx, ens,
                full != 0);
    __syncwarp();
  }
}

// The twigs above kMidCount: a group of 8 lanes per climb start computes its
// twig from the children, then climbs while it is the last child to arrive
// at the parent (fence, atomic, fence: the children's records are visible to
// the group that completes the parent).  list[start[6] .. start[7]).
__global__ void __launch_bounds__(128)
    k_net_top(const Geom* __restrict__ geom, double theta, int cap, double4* node_c,
              const int32_t* __restrict__ node_parent, int32_t* node_done,
              const int8_t* __restrict__ node_level, MixedNodes mx, Ensemble ens,
              const int32_t* __restrict__ start, const int32_t* __restrict__ list,
              int32_t* err) {
  const int b0 = start[6], b1 = start[7];
  const int lane = threadIdx.x & 31, j = lane & 7;
  const unsigned gm = 0xffu << (lane & 24);
  if (*((volatile int32_t*)err) & (kErrCapacity | kErrWalk)) return;
  const int ng = (gridDim.x * blockDim.x) >> 3;
  for (int k = b0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 3); k < b1; k += ng) {
    int t = list[k];
    const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, __ldg(&mx.first[t])) : 0;
    const double smax0 = geom[seg].smax0;
    for (int g = 0;; ++g) {
      if (g > kMaxLevel + 2) {
        if (j == 0) set_error(err, kErrWalk);
        break;
      }
      if (!net_twig8(t, j, gm, smax0, theta, cap, node_c, node_level, mx, err)) break;
      const int par = node_parent[t];
      int last = 0;
      if (j == 0 && par >= 0) {
        __threadfence();
        last = atomicSub(&node_done[par], 1) == 1;
      }
      if (!__shfl_sync(gm, last, lane & 24)) break;
      __threadfence();
      t = par;
    }
  }
}

// The net-charge moments of the combined tree (sort of the twigs into
// classes, direct sums, climb) once the topology (with the leaves' positions
// and the sorted copy xs) and the child tables exist.  Returns launches.
int net_moments(const BuildBuffers& b, int n, double theta, const Ensemble& ens, bool full,
                cudaStream_t st) {
  const int T = kNetThreads;
  const int NB = (b.cap + kNetBlockNodes - 1) / kNetBlockNodes;
  int32_t* cnt = b.mx.cls;                  // 7 NB class counts
  int32_t* off = b.mx.cls + 7 * NB;         // their exclusive scan
  int32_t* start = b.mx.lvl + 16;           // 8 class starts
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int gblk = NB < 4 * sms ? NB : 4 * sms;
  k_net_mark<<<gblk, T, 0, st>>>(b.bounds, b.cap, NB, b.node_pt, b.node_done, b.mx, cnt);
  k_net_scan<<<1, 1024, 0, st>>>(b.bounds, b.cap, NB, cnt, off, start);
  k_net_fill<<<gblk, T, 0, st>>>(b.bounds, b.cap, NB, b.node_pt, b.node_done, b.mx, off,
                                 b.mx.lvl_list);
  int g1 = (n / 2 + T - 1) / T;  // at most n - 1 twigs
  if (g1 > sms * 8) g1 = sms * 8;
  if (g1 < 1) g1 = 1;
  k_net_p2m_thread<<<g1, T, 0, st>>>(b.geom, theta, b.node_c, b.node_level, b.node_parent,
                                     b.mx, ens, start, b.mx.lvl_list, full ? 1 : 0, b.err);
  int g2 = (n / kSmallCount * 32 + T - 1) / T;
  if (g2 > sms * 8) g2 = sms * 8;
  if (g2 < 1) g2 = 1;
  k_net_p2m_warp<<<g2, T, 0, st>>>(b.geom, theta, b.node_c, b.node_level, b.node_parent,
                                   b.mx, ens, start, b.mx.lvl_list, full ? 1 : 0, b.err);
  k_net_top<<<sms, 128, 0, st>>>(b.geom, theta, b.cap, b.node_c, b.node_parent, b.node_done,
                                 b.node_level, b.mx, ens, start, b.mx.lvl_list, b.err);
  return 6;
}

}  // namespace tg
