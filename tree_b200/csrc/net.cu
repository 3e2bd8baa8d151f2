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
// node: particle count n, centroid X (the expansion centre), net charge Q,
// dipole D = sum q (x - X), second moment S = 1/2 sum q (x - X)(x - X)^T and
// the ion count.  Children are combined exactly (parallel axis):
//   d_c = X_c - X,  D = sum D_c + Q_c d_c,
//   S = sum S_c + (D_c d_c^T + d_c D_c^T)/2 + Q_c d_c d_c^T / 2.
// In a quasi-neutral plasma Q ~ 0 for large cells and the far field is the
// small net (dipole/quadrupole) field, so its truncation error is relative to
// that net field rather than to each species' monopole.
// Also the third moment T_ijk = sum q a_i a_j a_k (a = x - X), combined with
//   T += T_c + d_i S2_jk + d_j S2_ik + d_k S2_ij + d_i d_j D_k + d_i D_j d_k
//        + D_i d_j d_k + Q_c d_i d_j d_k      (S2 = 2 S of the child)
// -- the octupole the quadrupole expansion leaves out, whose size sets the
// error of accepting the cell.
// Also the fourth moment H_ijkl = sum q a_i a_j a_k a_l, combined with
//   H += H_c + 4 sym(d T_c) + 6 sym(d d S2_c) + 4 sym(d d d D_c) + Q_c d d d d
// (sym: the distinct index placements), for the hexadecapole far field.
// m64 per node (19 x double2): (n, Q) | (Dx, Dy) | (Dz, q_ion) | (Sxx, Syy) |
// (Szz, Sxy) | (Syz, Szx) | T in the order xxx yyy zzz xxy xxz xyy yyz xzz
// yzz xyz | H in the order xxxx yyyy zzzz xxxy xxxz xyyy yyyz xzzz yzzz xxyy
// xxzz yyzz xxyz xyyz xyzz, 0 (all raw, for the FP64 labels of the learned
// criterion).  The FP32
// copies the walk evaluates are trace-free, which drops every trace term from
// the far-field formula (phi = Q/r + D.d/r^3 + 3 d.S'.d/r^5 + 5/2 T'(d,d,d)/r^7):
// S' = S - tr(S)/3 I and T'_ijk = T_ijk - (d_ij V_k + d_ik V_j + d_jk V_i)/5
// with V_k = T_iik.  mom per node (3 x float4): (Q, Dx, Dy, Dz),
// (S'xx, S'yy, S'zz, Sxy), (Syz, Szx, trace S, q_ion); mom3 per node
// (3 x float4): (T'xxx, T'yyy, T'zzz, T'xxy), (T'xxz, T'xyy, T'yyz, T'xzz),
// (T'yzz, Txyz, |T'|_F, 0); mom4 per node (3 x float4): trace-free H'
// (xxxx, xxxy, xxxz, xxyy), (xxyz, xyyy, xyyz, yyyy), (yyyz, xxzz, xyzz,
// yyzz); geom (s, dx, n, |S'|_F).
// Leaves of the combined tree (one per sorted particle) and the sorted
// positions the walk reads.
__global__ void k_net_leaves(const double* __restrict__ x,
                             const uint32_t* __restrict__ vals,
                             const int8_t* __restrict__ L,
                             const int32_t* __restrict__ off, int n,
                             int n_el_charge, int cap, double4* node_c,
                             MixedNodes mx, Ensemble ens, int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (*((volatile int32_t*)err) & kErrCapacity) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  int ntw = hi > lo ? hi - lo : 0;
  int leaf = off[p] + ntw;
  if (leaf >= cap) return;
  uint32_t o = vals[p];
  // sorting keeps each cloud's index range, so p and o share the cloud
  const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, p) : 0;
  const bool ion = (int)o >= (ens.nseg > 0 ? __ldg(&ens.elec_end[seg]) : n_el_charge);
  const double q = ion ? 1.0 : -1.0;
  const double px = x[3 * (int64_t)o], py = x[3 * (int64_t)o + 1],
               pz = x[3 * (int64_t)o + 2];
  node_c[leaf] = make_double4(px, py, pz, -1.0);
  {
    double2* m = mx.m64 + kM64 * (int64_t)leaf;
    m[0] = make_double2(1.0, q);
    m[1] = make_double2(0.0, 0.0);
    m[2] = make_double2(0.0, ion ? 1.0 : 0.0);
#pragma unroll
    for (int u = 3; u < kM64; ++u) m[u] = make_double2(0.0, 0.0);
    float4* f3 = mx.mom3 + 3 * (int64_t)leaf;
    f3[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    f3[1] = make_float4(0.f, 0.f, 0.f, 0.f);
    f3[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4* f4 = mx.mom4 + 3 * (int64_t)leaf;
    f4[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    f4[1] = make_float4(0.f, 0.f, 0.f, 0.f);
    f4[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4* f = mx.mom + 3 * (int64_t)leaf;
    f[0] = make_float4((float)q, 0.f, 0.f, 0.f);
    f[1] = make_float4(0.f, 0.f, 0.f, 0.f);
    f[2] = make_float4(0.f, 0.f, 0.f, ion ? 1.f : 0.f);
    mx.geom[leaf] = make_float4(0.f, 0.f, 1.f, 0.f);
    mx.xs[p] = make_double4(px, py, pz, ion ? 1.0 : 0.0);
  }
}

// Net moments of twig `cur` from its children (all final): centroid, then
// Q, D, S, T and H about it by the parallel-axis rules, each summed over the
// children in pre-order (ascending octant digit, the order of the child
// table); writes the FP64 record and the trace-free FP32 copies.  One pass
// over the children per moment order keeps few accumulators live at a time
// (the children's records are re-read from L1/L2); the child indices come
// from one read of the child table, so the loads of all children are
// independent.
__device__ bool net_twig(int cur, double smax0, double theta, int cap,
                         double4* node_c, const int8_t* __restrict__ node_level,
                         MixedNodes mx, int32_t* err) {
  const double4 gc = ldcg_d4(&node_c[cur]);  // geometric centre (topology)
  int kid[8];
  {
    const int4* kk = reinterpret_cast<const int4*>(mx.kids + 8 * (int64_t)cur);
    const int4 k0 = __ldg(kk), k1 = __ldg(kk + 1);
    kid[0] = k0.x; kid[1] = k0.y; kid[2] = k0.z; kid[3] = k0.w;
    kid[4] = k1.x; kid[5] = k1.y; kid[6] = k1.z; kid[7] = k1.w;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (kid[j] >= cap || (kid[j] >= 0 && kid[j] <= cur)) {
      set_error(err, kErrWalk);
      return false;
    }
  // pass 1: count and centroid
  double nsum = 0.0, X0 = 0.0, X1 = 0.0, X2 = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = kid[j];
    if (c < 0) continue;
    const double4 cc = ldcg_d4(&node_c[c]);
    const double nc = __ldcg(mx.m64 + kM64 * (int64_t)c).x;
    nsum += nc;
    X0 += nc * cc.x;
    X1 += nc * cc.y;
    X2 += nc * cc.z;
  }
  X0 /= nsum;
  X1 /= nsum;
  X2 /= nsum;
  double2* m = mx.m64 + kM64 * (int64_t)cur;
  // pass 2: net charge, dipole and second moment about the centroid
  {
    double Q = 0, Dx = 0, Dy = 0, Dz = 0, qi = 0;
    double Sxx = 0, Syy = 0, Szz = 0, Sxy = 0, Syz = 0, Szx = 0;
#pragma unroll 1
    for (int j = 0; j < 8; ++j) {
      const int c = kid[j];
      if (c < 0) continue;
      const double4 cc = ldcg_d4(&node_c[c]);
      const double2* cm = mx.m64 + kM64 * (int64_t)c;
      const double2 a0 = __ldcg(cm), a1 = __ldcg(cm + 1), a2 = __ldcg(cm + 2),
                    a3 = __ldcg(cm + 3), a4 = __ldcg(cm + 4), a5 = __ldcg(cm + 5);
      const double qc = a0.y, dcx = a1.x, dcy = a1.y, dcz = a2.x;
      const double ex = cc.x - X0, ey = cc.y - X1, ez = cc.z - X2;
      Q += qc;
      qi += a2.y;
      Dx += dcx + qc * ex;
      Dy += dcy + qc * ey;
      Dz += dcz + qc * ez;
      Sxx += a3.x + dcx * ex + 0.5 * qc * ex * ex;
      Syy += a3.y + dcy * ey + 0.5 * qc * ey * ey;
      Szz += a4.x + dcz * ez + 0.5 * qc * ez * ez;
      Sxy += a4.y + 0.5 * (dcx * ey + ex * dcy) + 0.5 * qc * ex * ey;
      Syz += a5.x + 0.5 * (dcy * ez + ey * dcz) + 0.5 * qc * ey * ez;
      Szx += a5.y + 0.5 * (dcz * ex + ez * dcx) + 0.5 * qc * ez * ex;
    }
    const double a0 = X0 - gc.x, a1 = X1 - gc.y, a2 = X2 - gc.z;
    const double dx = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
    const int lev = node_level[cur];
    double smax = smax0;
    for (int l = 0; l < lev; ++l) smax = smax * 0.5;
    node_c[cur] = make_double4(X0, X1, X2, smax / theta + dx);
    m[0] = make_double2(nsum, Q);
    m[1] = make_double2(Dx, Dy);
    m[2] = make_double2(Dz, qi);
    m[3] = make_double2(Sxx, Syy);
    m[4] = make_double2(Szz, Sxy);
    m[5] = make_double2(Syz, Szx);
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
  // pass 3: third moment, parallel axis (T in the order xxx yyy zzz xxy xxz
  // xyy yyz xzz yzz xyz)
  {
    double T[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int j = 0; j < 8; ++j) {
      const int c = kid[j];
      if (c < 0) continue;
      const double4 cc = ldcg_d4(&node_c[c]);
      const double2* cm = mx.m64 + kM64 * (int64_t)c;
      const double2 a0 = __ldcg(cm), a1 = __ldcg(cm + 1), a2 = __ldcg(cm + 2),
                    a3 = __ldcg(cm + 3), a4 = __ldcg(cm + 4), a5 = __ldcg(cm + 5);
      const double qc = a0.y, dcx = a1.x, dcy = a1.y, dcz = a2.x;
      const double ex = cc.x - X0, ey = cc.y - X1, ez = cc.z - X2;
      const double S2xx = 2 * a3.x, S2yy = 2 * a3.y, S2zz = 2 * a4.x, S2xy = 2 * a4.y,
                   S2yz = 2 * a5.x, S2xz = 2 * a5.y;
      double Tc[10];
#pragma unroll
      for (int u = 0; u < 5; ++u) {
        const double2 t2 = __ldcg(cm + 6 + u);
        Tc[2 * u] = t2.x;
        Tc[2 * u + 1] = t2.y;
      }
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
    }
#pragma unroll
    for (int u = 0; u < 5; ++u) m[6 + u] = make_double2(T[2 * u], T[2 * u + 1]);
    // trace-free parts (order xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz)
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
  // pass 4: fourth moment, parallel axis: H += H_c + 4 sym(d T_c) + 6 sym(d d
  // S2_c) + 4 sym(d d d D_c) + Q_c d d d d (H in the order xxxx yyyy zzzz xxxy
  // xxxz xyyy yyyz xzzz yzzz xxyy xxzz yyzz xxyz xyyz xyzz)
  {
    double H[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int j = 0; j < 8; ++j) {
      const int c = kid[j];
      if (c < 0) continue;
      const double4 cc = ldcg_d4(&node_c[c]);
      const double2* cm = mx.m64 + kM64 * (int64_t)c;
      const double2 a0 = __ldcg(cm), a1 = __ldcg(cm + 1), a2 = __ldcg(cm + 2),
                    a3 = __ldcg(cm + 3), a4 = __ldcg(cm + 4), a5 = __ldcg(cm + 5);
      const double qc = a0.y, dcx = a1.x, dcy = a1.y, dcz = a2.x;
      const double ex = cc.x - X0, ey = cc.y - X1, ez = cc.z - X2;
      const double S2xx = 2 * a3.x, S2yy = 2 * a3.y, S2zz = 2 * a4.x, S2xy = 2 * a4.y,
                   S2yz = 2 * a5.x, S2xz = 2 * a5.y;
      const double2 t0 = __ldcg(cm + 6), t1 = __ldcg(cm + 7), t2 = __ldcg(cm + 8),
                    t3 = __ldcg(cm + 9), t4 = __ldcg(cm + 10);
      const double Txxx = t0.x, Tyyy = t0.y, Tzzz = t1.x, Txxy = t1.y, Txxz = t2.x,
                   Txyy = t2.y, Tyyz = t3.x, Txzz = t3.y, Tyzz = t4.x, Txyz = t4.y;
      double Hc[16];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const double2 h2 = __ldcg(cm + 11 + u);
        Hc[2 * u] = h2.x;
        Hc[2 * u + 1] = h2.y;
      }
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
    }
#pragma unroll
    for (int u = 0; u < 7; ++u) m[11 + u] = make_double2(H[2 * u], H[2 * u + 1]);
    m[18] = make_double2(H[14], 0.0);
    // trace-free H' = H - sym(delta C)/7 + sym(delta delta) tr C/35, C_kl = H_mmkl;
    // the walk's hexadecapole reads 12 components
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
  return true;
}

// Upward pass over the twigs in two launches.  "Small" twigs hold at most
// kSubCount particles and kSubNodes nodes (a child of a small twig is small);
// each maximal small subtree is completed by one warp: per-node counts of
// pending twig children in shared memory, a shared queue of ready twigs, and
// rounds in which the lanes complete every ready twig at once and release
// the parents whose last child they completed.  The twigs above count the
// twig children they wait for in global memory; the lane that completes a
// subtree root decrements its parent's count, and the last arrival completes
// the parent and climbs on (fence, atomic, fence: the children's records are
// visible to the thread that completes the parent).  The arithmetic per twig
// is net_twig's whichever lane runs it.
constexpr int kSubCount = 64;
constexpr int kSubNodes = 512;
constexpr int kNetWarps = 4;
constexpr int kNetBlocksPerSm = 8;

__device__ __forceinline__ bool net_small(int i, int cap, const int32_t* __restrict__ node_skip,
                                          const MixedNodes& mx) {
  int end = node_skip[i];
  if (end > cap) end = cap;
  return mx.count[i] <= kSubCount && end - i <= kSubNodes;
}

// Marks the pass: node_done[t] = twig children of each twig t above the small
// subtrees; list / *nlist: the roots of the maximal small subtrees.
__global__ void k_net_mark(const int32_t* __restrict__ bounds, int cap,
                           const int32_t* __restrict__ node_pt,
                           const int32_t* __restrict__ node_parent,
                           const int32_t* __restrict__ node_skip,
                           int32_t* node_done, MixedNodes mx, int32_t* list,
                           int32_t* nlist) {
  const int m = bounds[2] < cap ? bounds[2] : cap;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || node_pt[i] >= 0) return;  // twigs only
  if (!net_small(i, cap, node_skip, mx)) {
    const int4* kk = reinterpret_cast<const int4*>(mx.kids + 8 * (int64_t)i);
    const int4 k0 = kk[0], k1 = kk[1];
    const int kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
    int tw = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) tw += (kv[j] >= 0 && kv[j] < cap && node_pt[kv[j]] < 0) ? 1 : 0;
    node_done[i] = tw;
  } else {
    const int par = node_parent[i];
    if (par < 0 || !net_small(par, cap, node_skip, mx)) list[atomicAdd(nlist, 1)] = i;
  }
}

__global__ void __launch_bounds__(32 * kNetWarps, 4)
    k_net_subtrees(const Geom* __restrict__ geom, double theta, int cap,
                   double4* node_c, const int32_t* __restrict__ node_skip,
                   const int32_t* __restrict__ node_pt,
                   const int32_t* __restrict__ node_parent, int32_t* node_done,
                   const int8_t* __restrict__ node_level, MixedNodes mx,
                   Ensemble ens, const int32_t* __restrict__ list,
                   const int32_t* __restrict__ nlist, int32_t* cursor, int32_t* err) {
  __shared__ int32_t s_pend[kNetWarps][kSubNodes];  // pending twig children
  __shared__ int16_t s_queue[kNetWarps][kSubNodes];  // ready twigs (local index)
  __shared__ int32_t s_tail[kNetWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t* pend = s_pend[w];
  int16_t* queue = s_queue[w];
  const int total = *nlist;
  for (;;) {
    int k = 0;
    if (lane == 0) k = atomicAdd(cursor, 1);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= total) return;
    if (*((volatile int32_t*)err) & (kErrCapacity | kErrWalk)) return;
    const int r = list[k];
    int end = node_skip[r];
    if (end > cap) end = cap;
    const int nn = end - r;  // <= kSubNodes (a small subtree)
    const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, mx.first[r]) : 0;
    const double smax0 = geom[seg].smax0;
    for (int j = lane; j < nn; j += 32) pend[j] = 0;
    if (lane == 0) s_tail[w] = 0;
    __syncwarp();
    // pending counts: every twig below the root registers with its parent
    for (int j = lane + 1; j < nn; j += 32)
      if (__ldg(&node_pt[r + j]) < 0) atomicAdd(&pend[__ldg(&node_parent[r + j]) - r], 1);
    __syncwarp();
    // the first round: twigs whose children are all leaves (in index order)
    for (int j0 = 0; j0 < nn; j0 += 32) {
      const int j = j0 + lane;
      const bool ready = j < nn && __ldg(&node_pt[r + j]) < 0 && pend[j] == 0;
      const unsigned bm = __ballot_sync(0xffffffffu, ready);
      const int base = s_tail[w];
      if (ready) queue[base + __popc(bm & ((1u << lane) - 1u))] = (int16_t)j;
      __syncwarp();
      if (lane == 0) s_tail[w] = base + __popc(bm);
      __syncwarp();
    }
    // rounds: complete the ready twigs, release parents whose last child ends
    bool ok = true;
    int head = 0;
    for (int guard = 0; ; ++guard) {
      const int tail = s_tail[w];
      if (head >= tail || guard > kSubNodes) break;
      const int cnt = min(32, tail - head);
      __syncwarp();
      if (lane < cnt) {
        const int j = queue[head + lane];
        ok = net_twig(r + j, smax0, theta, cap, node_c, node_level, mx, err) && ok;
        if (j > 0) {
          const int pj = __ldg(&node_parent[r + j]) - r;
          if (atomicSub(&pend[pj], 1) == 1) queue[atomicAdd(&s_tail[w], 1)] = (int16_t)pj;
        } else if (ok) {
          // the subtree root: climb through the twigs above
          __threadfence();
          int par = node_parent[r];
          for (int g2 = 0; par >= 0; ++g2) {
            if (g2 > kMaxLevel + 2) {
              set_error(err, kErrWalk);
              break;
            }
            if (atomicSub(&node_done[par], 1) != 1) break;
            __threadfence();
            if (!net_twig(par, smax0, theta, cap, node_c, node_level, mx, err)) break;
            __threadfence();
            par = node_parent[par];
          }
        }
      }
      head += cnt;
      __syncwarp();
    }
    (void)ok;
    __syncwarp();
  }
}

// The net-moment pass of the combined tree: leaves, marking of the small
// subtrees, then the subtrees and the twigs above them.  Returns launches.
int net_moments(const BuildBuffers& b, const double* x, int n, int n_el, double theta,
                const Ensemble& ens, cudaStream_t st) {
  const int T = 256;
  const int gb = (n + T - 1) / T;
  const int gcap = (b.cap + T - 1) / T;
  k_net_leaves<<<gb, T, 0, st>>>(x, b.vals, b.L, b.off, n, n_el, b.cap, b.node_c,
                                 b.mx, ens, b.err);
  // lvl[0]: subtree roots listed, lvl[1]: their cursor
  cudaMemsetAsync(b.mx.lvl, 0, 2 * sizeof(int32_t), st);
  k_net_mark<<<gcap, T, 0, st>>>(b.bounds, b.cap, b.node_pt, b.node_parent, b.node_skip,
                                 b.node_done, b.mx, b.mx.lvl_list, b.mx.lvl);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int sgrid = (n + kSubCount - 1) / kSubCount;
  if (sgrid > sms * kNetBlocksPerSm) sgrid = sms * kNetBlocksPerSm;
  if (sgrid < 1) sgrid = 1;
  k_net_subtrees<<<sgrid, 32 * kNetWarps, 0, st>>>(b.geom, theta, b.cap, b.node_c,
                                                   b.node_skip, b.node_pt, b.node_parent,
                                                   b.node_done, b.node_level, b.mx, ens,
                                                   b.mx.lvl_list, b.mx.lvl, b.mx.lvl + 1,
                                                   b.err);
  return 3;
}

}  // namespace tg
