// walk_mixed.cu -- warp-group Barnes-Hut walk in mixed precision.
//
// The mixed path walks ONE combined tree of both species (net-charge moments
// about each cell's particle centroid, built bottom-up by k_net_subtrees).
// One warp owns a target group -- a contiguous sorted range of at most 32
// particles of either species inside one cell, built by k_groups -- and
// builds ONE interaction list for it:
//   * group MAC: a cell is accepted when rcrit = s/theta + dx (the reference
//     criterion, tree.f90:736-743) is below the distance from the cell's charge
//     centre to the group's bounding box, so every target of the group would
//     also accept it on its own;
//   * accepted cells go to a shared-memory ring of far-field (M2P) entries,
//     leaves and twigs with at most `bucket` particles go to a ring of
//     particle (P2P) entries, other twigs push their children on a per-warp
//     stack;
//   * every 32 entries the warp stages them in shared memory and each lane
//     evaluates them for its own target in FP32 (particle pairs two at a time
//     on the packed f32x2 pipeline).
// Precision: positions, the group centre and the MAC stay FP64.  Cells are
// evaluated in FP32 relative to the group centre; particle pairs use a
// two-float (hi + lo) split of the FP64 offsets, so a pair separation keeps
// ~1e-7 relative accuracy even for the closest e-i pairs.  Chunk sums of 32
// terms are added into Kahan-compensated per-lane accumulators.
// Far field: net monopole, dipole and trace-free quadrupole (octupole at order
// 3, hexadecapole at order 4) about the centroid -- the Coulomb expansion of
// tree.f90:744-779 carried to full subtree moments and further, for cells
// whose net charge nearly cancels; accepted cells far from the group go into
// the group's fourth-order local expansion (local.cuh), evaluated once per
// target.  Near field: erf-Kelbg (or the reference laws) for every particle
// pair.  With a trained model, cells the fixed test opens may be accepted by
// the learned criterion (mac.cuh, mac_batch below).
#include <cstdio>
#include "local.cuh"
#include "mac.cuh"
#include "walk_mixed.h"

namespace tg {

constexpr int kMxWarps = 8;
constexpr int kMxThreads = 32 * kMxWarps;
constexpr int kStackCap = 8192;   // node indices per warp
constexpr int kM2pRing = 64;      // power of two, > 31 + 32
constexpr int kLocRing = 64;      // power of two, > 31 + 32
constexpr int kLocStride = kLocCoef | 1;  // odd row stride of the coefficient rows
constexpr int kP2pRing = 512;     // power of two, > 31 + 32 * kMaxBucket
constexpr int kMaxBucket = 8;
constexpr int kMaxBlocksPerSm = 4;
// Blocks per SM the walk without RDF counts is compiled for: the fixed test
// at 3 (80 registers, 24 resident warps), the learned criterion at 2 (128
// registers, 16 warps): its candidate ring and budget make the 80-register
// build spill, which cost 13 % of its walk at N = 1M (23.1 against 20.4 ms),
// while the fixed test runs 5 % faster at 80 registers than at 128.
constexpr int kMinBlocksPerSm = 3;
constexpr int kMinBlocksPerSmLearned = 2;
// With RDF counts the walk runs one block of kRdfWarps per SM that keeps both
// histograms (2 x 10001 u32) in shared memory and adds them to the global
// bins once, when the block ends.
constexpr int kRdfWarps = 16;

constexpr int kCandRing = 64;     // power of two, > 31 + 32
constexpr int kCellF4 = 9;        // float4 per staged far-field cell (order 4)
constexpr int kPartF4 = 5;        // float4 per staged source pair (4 used + pad)

struct WarpSmem {
  int m2p[kM2pRing];
  int loc[kLocRing];       // far cells summed into the group's local expansion
  int p2p[kP2pRing];
  int cq_node[kCandRing];  // learned-MAC candidates waiting for a full batch
  // The far-field and pair staging areas (and the learned MAC's feature
  // rows, in `cell`) are used one at a time by the warp: one buffer.
  union {
    // staged cells, kCellF4 float4 each: (dx, dy, dz, Q), (Dx, Dy, Dz, q_ion),
    // (Sxx, Syy, Szz, Sxy), (Syz, Szx, Txxx, Tyyy), (Tzzz, Txxy, Txxz, Txyy),
    // (Tyyz, Txzz, Tyzz, Txyz), then for order 4 (Hxxxx, Hxxxy, Hxxxz, Hxxyy),
    // (Hxxyz, Hxyyy, Hxyyz, Hyyyy), (Hyyyz, Hxxzz, Hxyzz, Hyyzz) -- S, T and
    // H trace-free
    float4 cell[32 * kCellF4];
    // staged sources in pairs, kPartF4 float4 per pair: sources 2b and 2b+1
    // side by side, (nhx nhx' nhy nhy') (nhz nhz' q q') (nlx nlx' nly nly')
    // (nlz nlz' idx idx'): negated hi / lo offsets from the group centre,
    // charge, sorted index bits
    float4 part[16 * kPartF4];
    // local-expansion coefficients of up to 32 cells, one row per lane
    // (odd stride: conflict-free rows and columns)
    float loc_rows[32 * kLocStride];
  };
  // pair constants of the group's cloud: 1/lambda^2 (ee, ei, ii), 1/rs,
  // 1/lambda (ee, ei, ii)
  float pk[8];
  // the group's box: centre and half extents (read where used, so that they
  // hold no registers across the walk loop)
  double gx, gy, gz, bx, by, bz;
  double hl2;  // the group's squared half-diagonal (local-expansion test)
  // learned criterion, per group: log10 of the error budget (-inf: none),
  // and the cells sent to the network / kept on the fixed decision.  Kept
  // here rather than in registers, which the walk loop needs for its
  // evaluations.
  float lbud;
  unsigned n_mlp, n_fallback;
  double2 phi[32];  // per lane: unscaled potential (all sources, ion part)
};

__device__ __forceinline__ void phi_add(WarpSmem& sm, int lane, double all, double ion) {
  double2 p = sm.phi[lane];
  p.x += all;
  p.y += ion;
  sm.phi[lane] = p;
}

struct MixedArgs {
  const double4* __restrict__ node_c;
  const float4* __restrict__ mom;
  const int32_t* __restrict__ kids;
  const int32_t* __restrict__ first;
  const int32_t* __restrict__ count;
  const double4* __restrict__ xs;
  const uint32_t* __restrict__ order;
  const int32_t* __restrict__ bounds;
  const int2* __restrict__ groups;
  const int32_t* __restrict__ n_groups;
  int n, n_el;
  int32_t* control;
  int32_t* stack;
  int bucket;
  int p2p_max;  // accepted cells with at most this many particles go to P2P
  // accepted cells far from the group go to its local expansion: h / d <=
  // loc_eps, h the group's half-diagonal, d the distance from its centre to
  // the cell's centroid; loc_eps = 0: never
  double loc_eps2;
  int physics;
  float inv_lam2_ee, inv_lam2_ei, inv_lam2_ii;
  float inv_lam_ee, inv_lam_ei, inv_lam_ii;
  float rs_inv;
  float dx_ei_inv_f, dx_ii_inv_f;  // 1 / RDF bin widths
  double* f;
  double2* epot_part;
  uint32_t* rdf;
  unsigned long long* counters;
  int32_t* err;
  // learned acceptance
  const MlpPacked* packed;
  const float* fmin;
  const float* fmax;
  const float4* geom;
  const float4* mom3;
  const float4* mom4;
  // per cell: its part K of the pre-filter (mac.cuh) and the distance
  // s / rho_hi + dx below which its acceptance ratio s / (d - dx) exceeds
  // rho_hi (the learned criterion's band)
  const float2* mac_k;
  const float* margins;  // m_lo, m_hi, pre-filter coefficients c0..c4
  const double* f_prev;
  float eta_over_eps;
  float rho_lo, rho_hi;
  float lam_ei;
  // ensemble of clouds (nseg > 0): cloud ranges, roots, pair constants
  int nseg;
  const int32_t* ens_start;
  const int32_t* roots;
  const float4* cloud_pk;  // 2 per cloud, the layout of WarpSmem::pk
};

struct Acc {
  float sx, sy, sz, cx, cy, cz;  // Kahan sums of the unscaled force
  // The unscaled potential (all sources, ion part) is summed in FP64 in the
  // warp's shared memory, one slot per lane (WarpSmem::phi): it is touched
  // once per batch of 32 entries and need not hold registers in between.
};

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  float y = v - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  *total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - v;
}

__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------- M2P ----
// Net monopole Q, dipole D, trace-free second moment S (from 1/2 sum q a a^T)
// and, for ORDER 3, trace-free third moment T (from sum q a a a) about the
// cell centroid.  With d = target - centroid, r = |d|:
//   phi = Q/r + D.d/r^3 + 3 d.S.d/r^5 + 5/2 T(d,d,d)/r^7
//   -grad phi = g d - D/r^3 - 6 S d/r^5 - 7.5 T(.,d,d)/r^7,
//   g = Q/r^3 + 3 D.d/r^5 + 15 d.S.d/r^7 + 17.5 T(d,d,d)/r^9.
// About 50 flop per entry at ORDER 2, 100 at ORDER 3 (FMA = 2).  The ion part
// of phi for the Epot_e/Epot_i split is taken at monopole order (q_ion / r).
template <int ORDER>
__device__ __forceinline__ void eval_m2p(WarpSmem& sm, int head, int cnt,
                                         const MixedArgs& a, double Gx,
                                         double Gy, double Gz, float tx,
                                         float ty, float tz, int lane,
                                         Acc& acc) {
  if (lane < cnt) {
    int node = sm.m2p[(head + lane) & (kM2pRing - 1)];
    double4 c = ldg_d4(&a.node_c[node]);
    const float4* mp = a.mom + 3 * (int64_t)node;
    float4 m0 = __ldg(mp), m1 = __ldg(mp + 1), m2 = __ldg(mp + 2);
    float4* cl = sm.cell + kCellF4 * lane;
    cl[0] = make_float4((float)(c.x - Gx), (float)(c.y - Gy), (float)(c.z - Gz), m0.x);
    cl[1] = make_float4(m0.y, m0.z, m0.w, m2.w);
    cl[2] = m1;
    if (ORDER >= 3) {
      const float4* tp = a.mom3 + 3 * (int64_t)node;
      const float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
      cl[3] = make_float4(m2.x, m2.y, t0.x, t0.y);
      cl[4] = make_float4(t0.z, t0.w, t1.x, t1.y);
      cl[5] = make_float4(t1.z, t1.w, t2.x, t2.y);
    } else {
      cl[3] = make_float4(m2.x, m2.y, 0.f, 0.f);
    }
    if (ORDER >= 4) {
      const float4* hp = a.mom4 + 3 * (int64_t)node;
      cl[6] = __ldg(hp);
      cl[7] = __ldg(hp + 1);
      cl[8] = __ldg(hp + 2);
    }
  }
  __syncwarp();
  float fx = 0.f, fy = 0.f, fz = 0.f, pa = 0.f, pi = 0.f;
#pragma unroll 1
  for (int k = 0; k < cnt; ++k) {
    const float4* cl = sm.cell + kCellF4 * k;
    const float4 A = cl[0], B = cl[1], C = cl[2], E = cl[3];
    const float dx = tx - A.x, dy = ty - A.y, dz = tz - A.z;
    // accepted cells are farther than rcrit >= 0; the 1e-30 only guards a
    // zero-size cell against an FP32 distance of 0
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 1e-30f)));
    // Normalised form: the moments are contracted with the unit vector
    // n = d / r and scaled by powers of s = 1/r, so every intermediate is
    // bounded by n (a/r)^k -- escaped electrons millions of um away would
    // otherwise overflow T(d,d,d) ~ |T| r^3 while 1/r^7 underflows.
    const float s = rsqrtf(r2), s2 = s * s;
    const float nx = dx * s, ny = dy * s, nz = dz * s;
    // S n with S = [[Sxx,Sxy,Szx],[Sxy,Syy,Syz],[Szx,Syz,Szz]]
    const float Sx = fmaf(C.x, nx, fmaf(C.w, ny, E.y * nz));
    const float Sy = fmaf(C.w, nx, fmaf(C.y, ny, E.x * nz));
    const float Sz = fmaf(E.y, nx, fmaf(E.x, ny, C.z * nz));
    const float u = fmaf(nx, Sx, fmaf(ny, Sy, nz * Sz));
    const float Dn = fmaf(B.x, nx, fmaf(B.y, ny, B.z * nz));
    // r^2 (-grad phi) = gp n - s D - 6 s^2 S n - 7.5 s^3 T(., n, n),
    // gp = Q + 3 s D.n + 15 s^2 n.S.n + 17.5 s^3 T(n,n,n);
    // r phi = Q + s D.n + 3 s^2 n.S.n + 2.5 s^3 T(n,n,n)
    const float su = s * u;
    float gp = fmaf(s, fmaf(15.f, su, 3.f * Dn), A.w);
    float php = fmaf(s, fmaf(3.f, su, Dn), A.w);
    const float c5 = -6.f * s2;
    float gx = fmaf(c5, Sx, -s * B.x);
    float gy = fmaf(c5, Sy, -s * B.y);
    float gz = fmaf(c5, Sz, -s * B.z);
    if (ORDER >= 3) {
      const float4 T1 = cl[4], T2 = cl[5];
      // T order: xxx = E.z, yyy = E.w, zzz = T1.x, xxy = T1.y, xxz = T1.z,
      // xyy = T1.w, yyz = T2.x, xzz = T2.y, yzz = T2.z, xyz = T2.w.  T is
      // trace-free (T_iik = 0), so T_kzz = -T_kxx - T_kyy and each component
      // of T(., n, n) takes five terms with a = nx^2 - nz^2, b = ny^2 - nz^2
      const float zz = nz * nz;
      const float a2 = fmaf(nx, nx, -zz), b2 = fmaf(ny, ny, -zz);
      const float x2 = nx + nx, y2 = ny + ny;
      const float xy2 = x2 * ny, xz2 = x2 * nz, yz2 = y2 * nz;
      const float Tx = fmaf(E.z, a2, fmaf(T1.w, b2, fmaf(T1.y, xy2, fmaf(T1.z, xz2, T2.w * yz2))));
      const float Ty = fmaf(T1.y, a2, fmaf(E.w, b2, fmaf(T1.w, xy2, fmaf(T2.w, xz2, T2.x * yz2))));
      const float Tz = fmaf(T1.z, a2, fmaf(T2.x, b2, fmaf(T2.w, xy2, fmaf(T2.y, xz2, T2.z * yz2))));
      const float T3 = fmaf(nx, Tx, fmaf(ny, Ty, nz * Tz));
      const float s3 = s2 * s;
      const float s3T3 = s3 * T3;
      gp = fmaf(17.5f, s3T3, gp);
      php = fmaf(2.5f, s3T3, php);
      const float c7 = -7.5f * s3;
      gx = fmaf(c7, Tx, gx);
      gy = fmaf(c7, Ty, gy);
      gz = fmaf(c7, Tz, gz);
    }
    if (ORDER >= 4) {
      // hexadecapole: r^2 (-grad phi) += 39.375 s^4 H(n,n,n,n) n - 17.5 s^4
      // H(., n, n, n); r phi += 4.375 s^4 H(n,n,n,n) (phi = 35/8 H(d,d,d,d)
      // / r^9).  H is trace-free, so each component of H(., n, n, n) is a
      // combination of seven cubic harmonics P1..P7 of n; the z component
      // reads the three dependent components xxzz, xyzz, yyzz staged with
      // the others.
      const float4 H0 = cl[6], H1 = cl[7], H2 = cl[8];
      const float xx = nx * nx, yy = ny * ny, zz3 = 3.f * nz * nz;
      const float P1 = nx * (xx - zz3);
      const float P6 = ny * (yy - zz3);
      const float P2 = 3.f * ny * fmaf(nz, -nz, xx);
      const float P4 = 3.f * nx * fmaf(nz, -nz, yy);
      const float P3 = nz * fmaf(3.f, xx, -nz * nz);
      const float P7 = nz * fmaf(3.f, yy, -nz * nz);
      const float P5 = 6.f * nx * ny * nz;
      // (xxxx xxxy xxxz xxyy) (xxyz xyyy xyyz yyyy) (yyyz xxzz xyzz yyzz)
      const float Vx = fmaf(H0.x, P1, fmaf(H0.y, P2, fmaf(H0.z, P3, fmaf(H0.w, P4,
                       fmaf(H1.x, P5, fmaf(H1.y, P6, H1.z * P7))))));
      const float Vy = fmaf(H0.y, P1, fmaf(H0.w, P2, fmaf(H1.x, P3, fmaf(H1.y, P4,
                       fmaf(H1.z, P5, fmaf(H1.w, P6, H2.x * P7))))));
      const float Vz = fmaf(H0.z, P1, fmaf(H1.x, P2, fmaf(H2.y, P3, fmaf(H1.z, P4,
                       fmaf(H2.z, P5, fmaf(H2.x, P6, H2.w * P7))))));
      const float H4 = fmaf(nx, Vx, fmaf(ny, Vy, nz * Vz));
      const float s4 = s2 * s2;
      const float s4H = s4 * H4;
      gp = fmaf(39.375f, s4H, gp);
      php = fmaf(4.375f, s4H, php);
      const float c9 = -17.5f * s4;
      gx = fmaf(c9, Vx, gx);
      gy = fmaf(c9, Vy, gy);
      gz = fmaf(c9, Vz, gz);
    }
    fx = fmaf(s2, fmaf(gp, nx, gx), fx);
    fy = fmaf(s2, fmaf(gp, ny, gy), fy);
    fz = fmaf(s2, fmaf(gp, nz, gz), fz);
    pa = fmaf(s, php, pa);
    pi = fmaf(B.w, s, pi);
  }
  __syncwarp();
  kahan_add(acc.sx, acc.cx, fx);
  kahan_add(acc.sy, acc.cy, fy);
  kahan_add(acc.sz, acc.cz, fz);
  phi_add(sm, lane, (double)pa, (double)pi);
}

// The same far field two cells at a time on the packed FP32 (f32x2) pipeline:
// cells 2b and 2b+1 are staged side by side, so one 16-byte shared load gives
// two float2 operands and every multiply-add serves both cells.  Used where
// the walk runs with 128 registers per thread (the RDF layout: one 16-warp
// block per SM), which holds the doubled live state without spills.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

template <int ORDER>
__device__ __forceinline__ void eval_m2p_x2(WarpSmem& sm, int head, int cnt,
                                            const MixedArgs& a, double Gx, double Gy,
                                            double Gz, float tx, float ty, float tz,
                                            int lane, Acc& acc) {
  constexpr int kRows = ORDER >= 4 ? 9 : (ORDER == 3 ? 6 : 4);
  {
    // this lane's cell as kRows float4 rows (the layout of eval_m2p), or a
    // chargeless dummy far away past cnt
    float4 r[kRows];
    if (lane < cnt) {
      const int node = sm.m2p[(head + lane) & (kM2pRing - 1)];
      const double4 c = ldg_d4(&a.node_c[node]);
      const float4* mp = a.mom + 3 * (int64_t)node;
      const float4 m0 = __ldg(mp), m1 = __ldg(mp + 1), m2 = __ldg(mp + 2);
      r[0] = make_float4((float)(c.x - Gx), (float)(c.y - Gy), (float)(c.z - Gz), m0.x);
      r[1] = make_float4(m0.y, m0.z, m0.w, m2.w);
      r[2] = m1;
      if (ORDER >= 3) {
        const float4* tp = a.mom3 + 3 * (int64_t)node;
        const float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
        r[3] = make_float4(m2.x, m2.y, t0.x, t0.y);
        r[4] = make_float4(t0.z, t0.w, t1.x, t1.y);
        r[5] = make_float4(t1.z, t1.w, t2.x, t2.y);
      } else {
        r[3] = make_float4(m2.x, m2.y, 0.f, 0.f);
      }
      if (ORDER >= 4) {
        const float4* hp = a.mom4 + 3 * (int64_t)node;
        r[6] = __ldg(hp);
        r[7] = __ldg(hp + 1);
        r[8] = __ldg(hp + 2);
      }
    } else {
      r[0] = make_float4(1.0e6f, 1.0e6f, 1.0e6f, 0.f);
#pragma unroll
      for (int j = 1; j < kRows; ++j) r[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // pair block b = lane / 2: row j of both cells as (x x' y y') (z z' w w');
    // the even lane writes the first float4, the odd lane the second
    const bool odd = lane & 1;
    float4* blk = sm.cell + 2 * kCellF4 * (lane >> 1);
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const float s0 = odd ? r[j].x : r[j].z, s1 = odd ? r[j].y : r[j].w;
      const float p0 = __shfl_xor_sync(0xffffffffu, s0, 1);
      const float p1 = __shfl_xor_sync(0xffffffffu, s1, 1);
      blk[2 * j + (odd ? 1 : 0)] = odd ? make_float4(p0, r[j].z, p1, r[j].w)
                                       : make_float4(r[j].x, p0, r[j].y, p1);
    }
  }
  __syncwarp();
  const float2 tx2 = f2(tx), ty2 = f2(ty), tz2 = f2(tz);
  float2 fx = f2(0.f), fy = fx, fz = fx, pa = fx, pi = fx;
  const int npair = (cnt + 1) >> 1;
#pragma unroll 1
  for (int b = 0; b < npair; ++b) {
    const float4* bl = sm.cell + 2 * kCellF4 * b;
    float4 q = bl[0];
    const float2 Ax = make_float2(q.x, q.y), Ay = make_float2(q.z, q.w);
    q = bl[1];
    const float2 Az = make_float2(q.x, q.y), Q = make_float2(q.z, q.w);
    q = bl[2];
    const float2 Dx = make_float2(q.x, q.y), Dy = make_float2(q.z, q.w);
    q = bl[3];
    const float2 Dz = make_float2(q.x, q.y), Qi = make_float2(q.z, q.w);
    q = bl[4];
    const float2 Sxx = make_float2(q.x, q.y), Syy = make_float2(q.z, q.w);
    q = bl[5];
    const float2 Szz = make_float2(q.x, q.y), Sxy = make_float2(q.z, q.w);
    q = bl[6];
    const float2 Syz = make_float2(q.x, q.y), Szx = make_float2(q.z, q.w);
    const float2 dx = add2(tx2, make_float2(-Ax.x, -Ax.y));
    const float2 dy = add2(ty2, make_float2(-Ay.x, -Ay.y));
    const float2 dz = add2(tz2, make_float2(-Az.x, -Az.y));
    const float2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, f2(1e-30f))));
    const float2 s = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 s2 = mul2(s, s);
    const float2 nx = mul2(dx, s), ny = mul2(dy, s), nz = mul2(dz, s);
    const float2 Sx = fma2(Sxx, nx, fma2(Sxy, ny, mul2(Szx, nz)));
    const float2 Sy = fma2(Sxy, nx, fma2(Syy, ny, mul2(Syz, nz)));
    const float2 Sz = fma2(Szx, nx, fma2(Syz, ny, mul2(Szz, nz)));
    const float2 u = fma2(nx, Sx, fma2(ny, Sy, mul2(nz, Sz)));
    const float2 Dn = fma2(Dx, nx, fma2(Dy, ny, mul2(Dz, nz)));
    const float2 su = mul2(s, u);
    float2 gp = fma2(s, fma2(f2(15.f), su, mul2(f2(3.f), Dn)), Q);
    float2 php = fma2(s, fma2(f2(3.f), su, Dn), Q);
    const float2 c5 = mul2(f2(-6.f), s2);
    const float2 ms = make_float2(-s.x, -s.y);
    float2 gx = fma2(c5, Sx, mul2(ms, Dx));
    float2 gy = fma2(c5, Sy, mul2(ms, Dy));
    float2 gz = fma2(c5, Sz, mul2(ms, Dz));
    if (ORDER >= 3) {
      // (Syz Szx Txxx Tyyy) (Tzzz Txxy Txxz Txyy) (Tyyz Txzz Tyzz Txyz)
      q = bl[7];
      const float2 Txxx = make_float2(q.x, q.y), Tyyy = make_float2(q.z, q.w);
      q = bl[8];
      const float2 Txxy = make_float2(q.z, q.w);
      q = bl[9];
      const float2 Txxz = make_float2(q.x, q.y), Txyy = make_float2(q.z, q.w);
      q = bl[10];
      const float2 Tyyz = make_float2(q.x, q.y), Txzz = make_float2(q.z, q.w);
      q = bl[11];
      const float2 Tyzz = make_float2(q.x, q.y), Txyz = make_float2(q.z, q.w);
      const float2 zz = mul2(nz, nz);
      const float2 mzz = make_float2(-zz.x, -zz.y);
      const float2 a2 = fma2(nx, nx, mzz), b2 = fma2(ny, ny, mzz);
      const float2 x2 = add2(nx, nx), y2 = add2(ny, ny);
      const float2 xy2 = mul2(x2, ny), xz2 = mul2(x2, nz), yz2 = mul2(y2, nz);
      const float2 Tx = fma2(Txxx, a2, fma2(Txyy, b2, fma2(Txxy, xy2, fma2(Txxz, xz2, mul2(Txyz, yz2)))));
      const float2 Ty = fma2(Txxy, a2, fma2(Tyyy, b2, fma2(Txyy, xy2, fma2(Txyz, xz2, mul2(Tyyz, yz2)))));
      const float2 Tz = fma2(Txxz, a2, fma2(Tyyz, b2, fma2(Txyz, xy2, fma2(Txzz, xz2, mul2(Tyzz, yz2)))));
      const float2 T3 = fma2(nx, Tx, fma2(ny, Ty, mul2(nz, Tz)));
      const float2 s3T3 = mul2(mul2(s2, s), T3);
      gp = fma2(f2(17.5f), s3T3, gp);
      php = fma2(f2(2.5f), s3T3, php);
      const float2 c7 = mul2(f2(-7.5f), mul2(s2, s));
      gx = fma2(c7, Tx, gx);
      gy = fma2(c7, Ty, gy);
      gz = fma2(c7, Tz, gz);
    }
    if (ORDER >= 4) {
      // (xxxx xxxy xxxz xxyy) (xxyz xyyy xyyz yyyy) (yyyz xxzz xyzz yyzz)
      q = bl[12];
      const float2 H0 = make_float2(q.x, q.y), H1 = make_float2(q.z, q.w);
      q = bl[13];
      const float2 H2 = make_float2(q.x, q.y), H3 = make_float2(q.z, q.w);
      q = bl[14];
      const float2 H4 = make_float2(q.x, q.y), H5 = make_float2(q.z, q.w);
      q = bl[15];
      const float2 H6 = make_float2(q.x, q.y), H7 = make_float2(q.z, q.w);
      q = bl[16];
      const float2 H8 = make_float2(q.x, q.y), H9 = make_float2(q.z, q.w);
      q = bl[17];
      const float2 H10 = make_float2(q.x, q.y), H11 = make_float2(q.z, q.w);
      const float2 xx = mul2(nx, nx), yy = mul2(ny, ny);
      const float2 zz3 = mul2(f2(3.f), mul2(nz, nz));
      const float2 mnz = make_float2(-nz.x, -nz.y);
      const float2 P1 = mul2(nx, add2(xx, make_float2(-zz3.x, -zz3.y)));
      const float2 P6 = mul2(ny, add2(yy, make_float2(-zz3.x, -zz3.y)));
      const float2 P2 = mul2(mul2(f2(3.f), ny), fma2(nz, mnz, xx));
      const float2 P4 = mul2(mul2(f2(3.f), nx), fma2(nz, mnz, yy));
      const float2 P3 = mul2(nz, fma2(f2(3.f), xx, mul2(mnz, nz)));
      const float2 P7 = mul2(nz, fma2(f2(3.f), yy, mul2(mnz, nz)));
      const float2 P5 = mul2(mul2(f2(6.f), nx), mul2(ny, nz));
      const float2 Vx = fma2(H0, P1, fma2(H1, P2, fma2(H2, P3, fma2(H3, P4,
                        fma2(H4, P5, fma2(H5, P6, mul2(H6, P7)))))));
      const float2 Vy = fma2(H1, P1, fma2(H3, P2, fma2(H4, P3, fma2(H5, P4,
                        fma2(H6, P5, fma2(H7, P6, mul2(H8, P7)))))));
      const float2 Vz = fma2(H2, P1, fma2(H4, P2, fma2(H9, P3, fma2(H6, P4,
                        fma2(H10, P5, fma2(H8, P6, mul2(H11, P7)))))));
      const float2 H4n = fma2(nx, Vx, fma2(ny, Vy, mul2(nz, Vz)));
      const float2 s4 = mul2(s2, s2);
      const float2 s4H = mul2(s4, H4n);
      gp = fma2(f2(39.375f), s4H, gp);
      php = fma2(f2(4.375f), s4H, php);
      const float2 c9 = mul2(f2(-17.5f), s4);
      gx = fma2(c9, Vx, gx);
      gy = fma2(c9, Vy, gy);
      gz = fma2(c9, Vz, gz);
    }
    fx = fma2(s2, fma2(gp, nx, gx), fx);
    fy = fma2(s2, fma2(gp, ny, gy), fy);
    fz = fma2(s2, fma2(gp, nz, gz), fz);
    pa = fma2(s, php, pa);
    pi = fma2(Qi, s, pi);
  }
  __syncwarp();
  kahan_add(acc.sx, acc.cx, fx.x + fx.y);
  kahan_add(acc.sy, acc.cy, fy.x + fy.y);
  kahan_add(acc.sz, acc.cz, fz.x + fz.y);
  phi_add(sm, lane, (double)pa.x + (double)pa.y, (double)pi.x + (double)pi.y);
}

// -------------------------------------------------------------- local ----
// Up to 32 far cells, one per lane: each lane expands its cell's field about
// the group centre G (local.cuh) into its row of `loc_rows`; lanes 0..28 then
// add one coefficient each over the rows to their running sum `lsum`.  The
// group's targets evaluate the summed expansion once, after the walk.
template <int ORDER>
__device__ __forceinline__ void eval_local(WarpSmem& sm, int head, int cnt,
                                           const MixedArgs& a, double Gx, double Gy,
                                           double Gz, int lane, float& lsum) {
  constexpr int kStride = kLocStride;
  if (lane < cnt) {
    const int node = sm.loc[(head + lane) & (kLocRing - 1)];
    const double4 c = ldg_d4(&a.node_c[node]);
    CellMoments m;
    const float4* mp = a.mom + 3 * (int64_t)node;
    const float4 m0 = __ldg(mp), m1 = __ldg(mp + 1), m2 = __ldg(mp + 2);
    m.q = m0.x;
    m.d[0] = m0.y; m.d[1] = m0.z; m.d[2] = m0.w;
    m.s[0] = m1.x; m.s[1] = m1.y; m.s[2] = m1.z; m.s[3] = m1.w;
    m.s[4] = m2.x; m.s[5] = m2.y;
    m.q_ion = m2.w;
    if (ORDER >= 3) {
      const float4* tp = a.mom3 + 3 * (int64_t)node;
      const float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
      m.t[0] = t0.x; m.t[1] = t0.y; m.t[2] = t0.z; m.t[3] = t0.w;
      m.t[4] = t1.x; m.t[5] = t1.y; m.t[6] = t1.z; m.t[7] = t1.w;
      m.t[8] = t2.x; m.t[9] = t2.y;
    }
    if (ORDER >= 4) {
      const float4* hp = a.mom4 + 3 * (int64_t)node;
      const float4 h0 = __ldg(hp), h1 = __ldg(hp + 1), h2 = __ldg(hp + 2);
      m.h[0] = h0.x; m.h[1] = h0.y; m.h[2] = h0.z; m.h[3] = h0.w;
      m.h[4] = h1.x; m.h[5] = h1.y; m.h[6] = h1.z; m.h[7] = h1.w;
      m.h[8] = h2.x; m.h[9] = h2.y; m.h[10] = h2.z; m.h[11] = h2.w;
    }
    local_coefs<ORDER>((float)(Gx - c.x), (float)(Gy - c.y), (float)(Gz - c.z), m,
                       sm.loc_rows + kStride * lane);
  }
  __syncwarp();
  if (lane < kLocCoef) {
    float t = 0.f;
    for (int k = 0; k < cnt; ++k) t += sm.loc_rows[kStride * k + lane];
    lsum += t;
  }
  __syncwarp();
}

// ---------------------------------------------------------------- P2P ----
// Staged pair block (kPartF4 float4, sources 2b and 2b+1 side by side):
//   q0 (nhx nhx' nhy nhy')  q1 (nhz nhz' q q')  q2 (nlx nlx' nly nly')
//   q3 (nlz nlz' idx idx')
// negated hi / lo FP32 parts of each source's FP64 offset from the group
// centre, its charge (-1 electron, +1 ion; 0 for padding) and its sorted index.
//
// A pair's separation is formed from the hi parts alone.  Each hi part is
// within 2^-24 of its offset, so the separation r is within 2^-24 (2h + r)
// of the exact one (h the group's half-diagonal, which bounds the target's
// offset); for r^2 > h^2/32 that is below 7.3e-7 r.  Closer pairs -- a few in
// a thousand, among them every pair of the Kelbg core, the target itself and
// particles on one point -- are redone with hi + lo, whose FP32 roundings are
// relative to their own results, and only they need the source index.

// RDF counts of two pairs (e-i for every target, i-i for ion targets, as
// Search_Tree_ie/ei/ii bin them).  The bin is the FP32 distance r = r2 /
// sqrt(r2) (rsqrt within 2 ulp) over the bin width: within about 1e-6
// relative of the FP64 distance (see above), so a pair within that of a bin
// edge can land in the neighbouring bin; the FP64 path bins in FP64.
// s0 / s1: the source indices, or -1 when a pair was not close (it is then
// not the target).
template <int PHYS>
__device__ __forceinline__ void rdf_count2(const MixedArgs& a, uint32_t* hist, float2 r2,
                                           float2 rinv, float2 q, int s0, int s1,
                                           int p_self, int tsp) {
  const float tq = tsp ? 1.f : -1.f;
  const bool same0 = q.x == tq, same1 = q.y == tq;
  const float2 inv = make_float2(same0 ? a.dx_ii_inv_f : a.dx_ei_inv_f,
                                 same1 ? a.dx_ii_inv_f : a.dx_ei_inv_f);
  const float2 t = __fmul2_rn(__fmul2_rn(r2, rinv), inv);
  // counted pairs: a source (q != 0) of the other species, or an ion for an
  // ion target; never the target itself (Kelbg) or inside the same-species
  // cutoff (reference laws)
  const bool ok0 = q.x != 0.f && (!same0 || tsp == 1) &&
                   (PHYS == 1 ? s0 != p_self : (same0 ? r2.x > 0.01f : true));
  const bool ok1 = q.y != 0.f && (!same1 || tsp == 1) &&
                   (PHYS == 1 ? s1 != p_self : (same1 ? r2.y > 0.01f : true));
  // r2 = 0 (distinct particles on one point): bin 0
  const float t0 = r2.x > 0.f ? t.x : 0.f, t1 = r2.y > 0.f ? t.y : 0.f;
  if (ok0 && t0 < (float)kRdfBins) atomicAdd(&hist[(same0 ? kRdfBins : 0) + (int)t0], 1u);
  if (ok1 && t1 < (float)kRdfBins) atomicAdd(&hist[(same1 ? kRdfBins : 0) + (int)t1], 1u);
}

// One source against this lane's target with every case of the pair laws:
// "special" pairs leave the plain Coulomb law -- the target itself (r = 0),
// pairs inside the Kelbg core (exp(-x^2) still visible in FP32), and for the
// reference laws same-species pairs inside the r^2 <= 0.01 cutoff and e-i
// pairs where exp(-r/rs) is visible.
template <int PHYS>
__device__ __forceinline__ void p2p_one(const WarpSmem& sm, float r2, float dx, float dy,
                                        float dz, float ssign, int s, int p_self, int tsp,
                                        float& fx, float& fy, float& fz, float& pa,
                                        float& pq) {
  const bool same = ssign == (tsp ? 1.f : -1.f);
  const float il2_same = PHYS == 1 ? (tsp ? sm.pk[2] : sm.pk[0]) : 0.f;
  const float il_same = PHYS == 1 ? (tsp ? sm.pk[6] : sm.pk[4]) : 0.f;
  const float il2_ei = sm.pk[1], il_ei = sm.pk[5], rs_inv = sm.pk[3];
  bool special;
  if (PHYS == 1) special = r2 * (same ? il2_same : il2_ei) < 40.f;
  else special = same ? !(r2 > 0.01f) : r2 * (rs_inv * rs_inv) < 400.f;
  float fs, ph;
  if (!special) {
    const float rinv = rsqrtf(r2);
    fs = ssign * rinv * rinv * rinv;
    ph = ssign * rinv;
  } else {
    fs = 0.f;
    ph = 0.f;
    if (PHYS == 1) {
      if (s != p_self) {
        const float il = same ? il_same : il_ei;
        const float sqrtpi = 1.77245385f;
        float ve;
        if (r2 > 0.f) {
          const float r = sqrtf(r2);
          const float ri = 1.f / r;
          const float x2 = r2 * il * il;
          const float g = -expm1f(-x2);
          fs = ssign * g * ri * ri * ri;
          ve = g * ri + sqrtpi * erfcf(r * il) * il;
        } else {
          ve = sqrtpi * il;  // distinct particles on one point: V(0)
        }
        ph = ssign * ve;
      }
    } else if (!same) {
      float ve;
      if (r2 > 0.f) {
        const float r = sqrtf(r2);
        const float ri = 1.f / r;
        const float e = expf(-r * rs_inv);
        const float g = ri - e * (ri + rs_inv);
        fs = ssign * g * ri * ri;
        ve = (1.f - e) * ri;
      } else {
        ve = rs_inv;  // r -> 0 limit of (1 - exp(-r/rs))/r
      }
      ph = ssign * ve;
    }  // same species inside the cutoff (and the target itself): nothing
  }
  fx = fmaf(fs, dx, fx);
  fy = fmaf(fs, dy, fy);
  fz = fmaf(fs, dz, fz);
  pa += ph;
  pq = fmaf(ssign, ph, pq);
}

// Pair interactions of up to 32 staged sources with this lane's target, two
// sources per packed FP32 (f32x2) instruction.  The common pair is plain
// Coulomb from the hi parts; a close pair (r^2 <= close2) is redone with the
// exact offsets, and a pair with a special member goes through p2p_one.
template <int PHYS, bool RDF>
__device__ __forceinline__ void eval_p2p(WarpSmem& sm, int head, int cnt,
                                         const MixedArgs& a, double Gx,
                                         double Gy, double Gz, float thx,
                                         float thy, float thz, float tlx,
                                         float tly, float tlz, float close2,
                                         int p_self, int tsp, bool act, int lane,
                                         uint32_t* hist, Acc& acc) {
  {
    // this lane's source (or, past cnt, a chargeless dummy 10^6 um away)
    float v[8];
    if (lane < cnt) {
      const int s = sm.p2p[(head + lane) & (kP2pRing - 1)];
      const double4 xs = a.xs[s];
      const double rx = Gx - xs.x, ry = Gy - xs.y, rz = Gz - xs.z;
      const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
      v[0] = hx; v[1] = hy; v[2] = hz; v[3] = xs.w > 0.5 ? 1.f : -1.f;
      v[4] = (float)(rx - (double)hx); v[5] = (float)(ry - (double)hy);
      v[6] = (float)(rz - (double)hz); v[7] = __int_as_float(s);
    } else {
      v[0] = v[1] = v[2] = 1.0e6f;
      v[3] = 0.f;
      v[4] = v[5] = v[6] = 0.f;
      v[7] = __int_as_float(-1);
    }
    const bool odd = lane & 1;
    float2* pb = reinterpret_cast<float2*>(sm.part + kPartF4 * (lane >> 1)) + (odd ? 1 : 0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float lo = v[2 * j], hi = v[2 * j + 1];
      const float o_lo = __shfl_xor_sync(0xffffffffu, lo, 1);
      const float o_hi = __shfl_xor_sync(0xffffffffu, hi, 1);
      pb[2 * j] = odd ? make_float2(o_hi, hi) : make_float2(lo, o_lo);
    }
  }
  __syncwarp();
  // the source charge that makes a pair "same species" for this target, and
  // the FP32 screening constants of the common-path test
  const float tq = tsp ? 1.f : -1.f;
  const float il2_to_e = PHYS == 1 ? (tsp ? sm.pk[1] : sm.pk[0]) : 0.f;  // electron source
  const float il2_to_i = PHYS == 1 ? (tsp ? sm.pk[2] : sm.pk[1]) : 0.f;  // ion source
  const float rs2 = sm.pk[3] * sm.pk[3];
  const float2 thx2 = make_float2(thx, thx), thy2 = make_float2(thy, thy), thz2 = make_float2(thz, thz);
  float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx, pa = fx, pq = fx;
  const int npair = (cnt + 1) >> 1;
  for (int b = 0; b < npair; ++b) {
    const float4* blk = sm.part + kPartF4 * b;
    const float4 q0 = blk[0], q1 = blk[1];
    const float2 q = make_float2(q1.z, q1.w);  // source charges: -1 e, +1 ion
    float2 dx = __fadd2_rn(thx2, make_float2(q0.x, q0.y));
    float2 dy = __fadd2_rn(thy2, make_float2(q0.z, q0.w));
    float2 dz = __fadd2_rn(thz2, make_float2(q1.x, q1.y));
    float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    int s0 = -1, s1 = -1;
    if (r2.x <= close2 || r2.y <= close2) {
      // close pair: the exact offsets (hi + lo) and the source indices
      const float4 q2 = blk[2], q3 = blk[3];
      dx = __fadd2_rn(__fadd2_rn(thx2, make_float2(q0.x, q0.y)),
                      __fadd2_rn(make_float2(tlx, tlx), make_float2(q2.x, q2.y)));
      dy = __fadd2_rn(__fadd2_rn(thy2, make_float2(q0.z, q0.w)),
                      __fadd2_rn(make_float2(tly, tly), make_float2(q2.z, q2.w)));
      dz = __fadd2_rn(__fadd2_rn(thz2, make_float2(q1.x, q1.y)),
                      __fadd2_rn(make_float2(tlz, tlz), make_float2(q3.x, q3.y)));
      r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
      s0 = __float_as_int(q3.z);
      s1 = __float_as_int(q3.w);
    }
    bool sp0, sp1;
    if (PHYS == 1) {
      sp0 = r2.x * (q.x < 0.f ? il2_to_e : il2_to_i) < 40.f;
      sp1 = r2.y * (q.y < 0.f ? il2_to_e : il2_to_i) < 40.f;
    } else {
      sp0 = q.x == tq ? !(r2.x > 0.01f) : r2.x * rs2 < 400.f;
      sp1 = q.y == tq ? !(r2.y > 0.01f) : r2.y * rs2 < 400.f;
    }
    const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    if (!(sp0 || sp1)) {
      const float2 ph = __fmul2_rn(q, rinv);
      const float2 fs = __fmul2_rn(ph, __fmul2_rn(rinv, rinv));
      fx = __ffma2_rn(fs, dx, fx);
      fy = __ffma2_rn(fs, dy, fy);
      fz = __ffma2_rn(fs, dz, fz);
      pa = __fadd2_rn(pa, ph);
      pq = __ffma2_rn(q, ph, pq);
    } else {
      p2p_one<PHYS>(sm, r2.x, dx.x, dy.x, dz.x, q.x, s0, p_self, tsp,
                    fx.x, fy.x, fz.x, pa.x, pq.x);
      p2p_one<PHYS>(sm, r2.y, dx.y, dy.y, dz.y, q.y, s1, p_self, tsp,
                    fx.y, fy.y, fz.y, pa.y, pq.y);
    }
    if (RDF && act) rdf_count2<PHYS>(a, hist, r2, rinv, q, s0, s1, p_self, tsp);
  }
  __syncwarp();
  kahan_add(acc.sx, acc.cx, fx.x + fx.y);
  kahan_add(acc.sy, acc.cy, fy.x + fy.y);
  kahan_add(acc.sz, acc.cz, fz.x + fz.y);
  const double pad = (double)pa.x + (double)pa.y, pqd = (double)pq.x + (double)pq.y;
  phi_add(sm, lane, pad, 0.5 * (pad + pqd));  // ion sources: (all + charge-weighted) / 2
}

// Squared distance from a cell's centroid to the group's box, in an
// operation order pinned against contraction: the network batch recomputes
// it for its candidates and must see the value the walk's test saw.
__device__ __forceinline__ double box_dist2(const double4& c, const WarpSmem& sm) {
  const double ex = fmax(fabs(c.x - sm.gx) - sm.bx, 0.0);
  const double ey = fmax(fabs(c.y - sm.gy) - sm.by, 0.0);
  const double ez = fmax(fabs(c.z - sm.gz) - sm.bz, 0.0);
  return __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
}

// ------------------------------------------------------ learned MAC ----
// One batch of queued candidates (lane < nb holds one) through the network.
// Returns 1 (accept) or 3 (open) for a candidate, 0 otherwise, plus 4 when
// its features fell outside the training range (the fixed decision, open,
// stands).  Out of line: it runs once per 32 candidates, and the network's
// fragments then take no registers from the walk loop around the call.
// A candidate's distance d and budget B = log10(budget d^2 / n) (the label's
// units) are recomputed here as the walk's test formed them.
__device__ __noinline__ int mac_batch(const double4* __restrict__ node_c,
                                      const float4* __restrict__ geom,
                                      const float4* __restrict__ mom,
                                      const float4* __restrict__ mom3, WarpSmem& sm,
                                      const MlpPacked* mlp, const float* frange, int node,
                                      bool cand, float n_act, int lane) {
  float* feat = reinterpret_cast<float*>(sm.cell) + lane * kMacFeatures;
  float cand_B = 0.f;
  if (cand) {
    const double4 c = ldg_d4(&node_c[node]);
    const float4 g4 = __ldg(&geom[node]);
    const float ddf = sqrtf((float)box_dist2(c, sm));
    cand_B = sm.lbud + 2.f * __log10f(ddf) - log10f(g4.z);
    const float4* mp = mom + 3 * (int64_t)node;
    const float4* tp = mom3 + 3 * (int64_t)node;
    mac_features(c.x, c.y, c.z, g4, __ldg(mp), __ldg(mp + 1), __ldg(mp + 2), __ldg(tp),
                 __ldg(tp + 1), __ldg(tp + 2), sm.gx, sm.gy, sm.gz, (float)sqrt(sm.hl2), ddf,
                 n_act, feat);
  } else {
#pragma unroll
    for (int k = 0; k < kMacFeatures; ++k) feat[k] = 0.f;
  }
  // range check on the raw features before the network normalises them
  bool in_range = true;
#pragma unroll
  for (int k = 0; k < kMacFeatures; ++k)
    in_range = in_range && feat[k] >= frange[k] && feat[k] <= frange[kMacFeatures + k];
  __syncwarp();
  const float y = mlp_forward_warp(reinterpret_cast<float*>(sm.cell), *mlp, lane);
  if (!cand) return 0;
  // predicted |dF| = 10^y * n / d^2 against the group's budget; out of the
  // training range the fixed-theta decision (open) stands
  return ((in_range && y <= cand_B) ? 1 : 3) | (in_range ? 0 : 4);
}

// Per cell, for the nodes [0, bounds[2]) of this build: its part K of the
// learned pre-filter (mac_node_term) and the distance s / rho_hi + dx inside
// which it lies outside the criterion's band.  Leaves are never tested; their
// records are not read.
__global__ void k_mac_node_terms(const float4* __restrict__ geom,
                                 const float4* __restrict__ mom3,
                                 const int32_t* __restrict__ bounds,
                                 const float* __restrict__ margins, float inv_rho_hi,
                                 float2* __restrict__ mac_k) {
  const int end = bounds[2];
  float c[kEstCoef];
#pragma unroll
  for (int k = 0; k < kEstCoef; ++k) c[k] = __ldg(&margins[2 + k]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    const float4 g4 = __ldg(&geom[i]);
    mac_k[i] = make_float2(mac_node_term(g4, __ldg(&mom3[3 * (int64_t)i + 2]).z, c),
                           fmaf(g4.x, inv_rho_hi, g4.y));
  }
}

// --------------------------------------------------------------- walk ----
// Dynamic shared memory: WarpSmem per warp, then (learned MAC only) the
// packed network and the features' training range, then (RDF only) the two
// block histograms.
constexpr size_t walk_learned_bytes() {
  return (sizeof(MlpPacked) + sizeof(float) * (2 * kMacFeatures + 8) + 15) / 16 * 16;
}
template <bool LEARNED, bool RDF>
constexpr size_t walk_smem_bytes() {
  return sizeof(WarpSmem) * (RDF ? kRdfWarps : kMxWarps) + (LEARNED ? walk_learned_bytes() : 0) +
         (RDF ? sizeof(uint32_t) * 2 * kRdfBins : 0);
}

// the largest variant must fit one block's opt-in shared memory (227 KB)
static_assert(walk_smem_bytes<true, true>() <= 232448, "walk shared memory over 227 KB");
static_assert(walk_smem_bytes<true, false>() * kMinBlocksPerSm <= 233472 - 3 * 1024,
              "three walk blocks no longer fit one SM");

template <int PHYS, bool RDF, bool LEARNED, int ORDER>
__global__ void __launch_bounds__(RDF ? 32 * kRdfWarps : kMxThreads,
                                  RDF ? 1 : (LEARNED ? kMinBlocksPerSmLearned : kMinBlocksPerSm))
    k_walk_mixed(MixedArgs a) {
  constexpr int kW = RDF ? kRdfWarps : kMxWarps;
  extern __shared__ float4 dyn_smem[];
  WarpSmem* smem = reinterpret_cast<WarpSmem*>(dyn_smem);
  unsigned char* tail = reinterpret_cast<unsigned char*>(smem + kW);
  MlpPacked* mlp = reinterpret_cast<MlpPacked*>(tail);
  uint32_t* hist = reinterpret_cast<uint32_t*>(tail + (LEARNED ? walk_learned_bytes() : 0));
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WarpSmem& sm = smem[wib];
  if (RDF) {
    for (int i = threadIdx.x; i < 2 * kRdfBins; i += blockDim.x) hist[i] = 0u;
    __syncthreads();
  }
  if (LEARNED) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.packed);
    uint32_t* dst = reinterpret_cast<uint32_t*>(mlp);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  // training range of the features (fmin | fmax), then m_lo, m_hi and the
  // pre-filter coefficients, shared by the block
  float* frange = reinterpret_cast<float*>(mlp + 1);
  const float* fmodel = frange + 2 * kMacFeatures;
  if (LEARNED) {
    if (threadIdx.x < kMacFeatures) {
      frange[threadIdx.x] = __ldg(&a.fmin[threadIdx.x]);
      frange[kMacFeatures + threadIdx.x] = __ldg(&a.fmax[threadIdx.x]);
    }
    if (threadIdx.x < 2 + kEstCoef)
      frange[2 * kMacFeatures + threadIdx.x] = __ldg(&a.margins[threadIdx.x]);
    __syncthreads();
  }
  const int gwarp = blockIdx.x * kW + wib;
  int32_t* stack = a.stack + (int64_t)gwarp * kStackCap;
  const unsigned lt = (1u << lane) - 1u;
  if (*((volatile int32_t*)a.err) & (kErrCapacity | kErrDepth | kErrNonFinite)) return;
  const int root_end = a.bounds[2];  // combined tree: nodes [0, root_end)
  const int ngroups = *a.n_groups;
  int max_stack = 0;
  while (root_end > 0) {
    int g = 0;
    if (lane == 0) g = atomicAdd(&a.control[0], 1);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= ngroups) break;
    const int2 grp = a.groups[g];
    const int p0 = grp.x, n_act = grp.y;
    const bool act = lane < n_act;
    const int pt = p0 + (act ? lane : n_act - 1);
    const double4 xt = a.xs[pt];
    const int tsp = xt.w > 0.5 ? 1 : 0;  // this lane's target species
    const double mnx = warp_min_d(xt.x), mny = warp_min_d(xt.y), mnz = warp_min_d(xt.z);
    const double mxx = warp_max_d(xt.x), mxy = warp_max_d(xt.y), mxz = warp_max_d(xt.z);
    const double Gx = 0.5 * (mnx + mxx), Gy = 0.5 * (mny + mxy), Gz = 0.5 * (mnz + mxz);
    const double hx = 0.5 * (mxx - mnx), hy = 0.5 * (mxy - mny), hz = 0.5 * (mxz - mnz);
    const double rtx = xt.x - Gx, rty = xt.y - Gy, rtz = xt.z - Gz;
    const float thx = (float)rtx, thy = (float)rty, thz = (float)rtz;
    const float tlx = (float)(rtx - (double)thx), tly = (float)(rty - (double)thy),
                tlz = (float)(rtz - (double)thz);
    // pairs closer than h / sqrt(32) (h the group's half-diagonal) take the
    // exact offsets (eval_p2p)
    const double hl2 = hx * hx + hy * hy + hz * hz;
    const float close2 = (float)(hl2 * (1.0 / 32.0));
    if (lane == 0) {
      sm.hl2 = hl2;
      sm.gx = Gx;
      sm.gy = Gy;
      sm.gz = Gz;
      sm.bx = hx;
      sm.by = hy;
      sm.bz = hz;
    }
    Acc acc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    sm.phi[lane] = make_double2(0.0, 0.0);
    // error budget of the learned MAC: eta * min |F_prev| / eps over the group
    if (LEARNED) {
      const int64_t o = a.order[pt];
      const double fx = a.f_prev[3 * o], fy = a.f_prev[3 * o + 1], fz = a.f_prev[3 * o + 2];
      float fm = act ? (float)sqrt(fx * fx + fy * fy + fz * fz) : 3.0e38f;
      for (int o2 = 16; o2 > 0; o2 >>= 1) fm = fminf(fm, __shfl_xor_sync(0xffffffffu, fm, o2));
      const float budget = a.eta_over_eps * fm;
      if (lane == 0) {
        sm.lbud = budget > 0.f ? log10f(budget) : -INFINITY;
        sm.n_mlp = 0u;
        sm.n_fallback = 0u;
      }
    }
    int ssize = 1;
    // the group's tree: its cloud's root and pair constants
    int root = 0;
    if (a.nseg > 0) {
      int c = 0;
      if (lane == 0) {
        int lo = 0, hi = a.nseg - 1;  // largest c with start[c] <= p0
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (__ldg(&a.ens_start[mid]) <= p0) lo = mid;
          else hi = mid - 1;
        }
        c = lo;
      }
      c = __shfl_sync(0xffffffffu, c, 0);
      root = __ldg(&a.roots[c]);
      if (lane < 8) sm.pk[lane] = __ldg(reinterpret_cast<const float*>(a.cloud_pk + 2 * c) + lane);
    } else if (lane == 0) {
      sm.pk[0] = a.inv_lam2_ee;
      sm.pk[1] = a.inv_lam2_ei;
      sm.pk[2] = a.inv_lam2_ii;
      sm.pk[3] = a.rs_inv;
      sm.pk[4] = a.inv_lam_ee;
      sm.pk[5] = a.inv_lam_ei;
      sm.pk[6] = a.inv_lam_ii;
      sm.pk[7] = 0.f;
    }
    if (lane == 0) stack[0] = root;
    __syncwarp();
    int m2h = 0, m2t = 0, p2h = 0, p2t = 0;  // ring heads/tails (warp-uniform)
    int lch = 0, lct = 0;                    // local-expansion ring
    float lsum = 0.f;  // lanes 0..19: one summed coefficient of the local expansion
    bool overflow = false;
    int cqh = 0, cqt = 0;  // learned-MAC candidate ring (warp-uniform)
    while (ssize > 0 || cqt > cqh) {
      int node = -1;
      int action = 0, pfirst = 0, pcnt = 0;  // 1 far field, 2 particles, 3 open
      if (LEARNED && (cqt - cqh >= 32 || (ssize == 0 && cqt > cqh))) {
        // ---- a batch of queued candidates goes through the network ----
        const int nb = min(32, cqt - cqh);
        const bool cand = lane < nb;
        if (cand) node = sm.cq_node[(cqh + lane) & (kCandRing - 1)];
        cqh += nb;
        __syncwarp();
        const int r = mac_batch(a.node_c, a.geom, a.mom, a.mom3, sm, mlp, frange, node, cand,
                                (float)n_act, lane);
        if (cand) action = r & 3;  // candidates exceed a bucket: accept or open
        const unsigned fbm = __ballot_sync(0xffffffffu, (r & 4) != 0);
        if (lane == 0) {
          sm.n_mlp += (unsigned)nb;
          sm.n_fallback += (unsigned)__popc(fbm);
        }
      } else {
        // ---- a batch of nodes from the stack ----
        const int nb = min(32, ssize);
        node = lane < nb ? stack[ssize - 1 - lane] : -1;
        ssize -= nb;
        __syncwarp();
        bool cand = false;  // queued for the learned MAC
        if (node >= 0) {
          // the particle range and (learned criterion) the cell's pre-filter
          // record depend on the node index alone: issued with node_c, so a
          // batch waits for one round of loads instead of two or three
          const double4 c = ldg_d4(&a.node_c[node]);
          const int cnt = __ldg(&a.count[node]);
          const int fst = __ldg(&a.first[node]);
          const float2 kr = LEARNED ? __ldg(&a.mac_k[node]) : make_float2(0.f, 0.f);
          if (c.w < 0.0) {
            action = 2;
            pfirst = fst;
            pcnt = 1;
          } else {
            // group MAC: rcrit below the distance from the centroid to the box
            const double d2 = box_dist2(c, sm);
            bool accept = c.w * c.w < d2;  // the fixed-theta test
            if (LEARNED && !accept) {
              // learned criterion, on top of the fixed test: a cell the fixed
              // test opens is accepted anyway when its predicted acceptance
              // error is within the group's budget.  rho = s / (d - dx) places
              // it against the training band; est is the fitted log-linear
              // estimate of the label (mac.cuh) and B the budget in the same
              // units.  Cells whose estimate is clearly on one side of B
              // (training quantiles m_lo, m_hi of label - est) are decided at
              // once; the rest are queued for the network.  Only cells that
              // would otherwise open into more than a bucket of particle
              // pairs are worth a far-field evaluation.
              // rho = s / (d - dx) <= rho_hi  <=>  d >= s / rho_hi + dx
              const float d2f = (float)d2;
              if (d2f >= kr.y * kr.y && cnt > a.bucket) {
                const float ddf = sqrtf(d2f);
                // est - B = K - log10(budget) - (2 + c0) log10(d); no
                // budget: log10(budget) = -inf, never accepted or queued
                const float lb = sm.lbud, l10d = __log10f(ddf);
                const float eb = fmaf(-(2.f + fmodel[2]), l10d, kr.x - lb);
                if (eb + fmodel[1] <= 0.f) {
                  accept = true;
                } else if (eb + fmodel[0] <= 0.f) {
                  cand = true;
                }
              }
            }
            // a small accepted cell is cheaper and exact as particle pairs: an
            // M2P costs about as much as p2p_max pair interactions
            if (accept && cnt <= a.p2p_max) {
              action = 2;
              pfirst = fst;
              pcnt = cnt;
            } else if (accept) {
              action = 1;
              if (a.loc_eps2 > 0.0) {
                // far from the group: summed into its local expansion
                const double ux = c.x - sm.gx, uy = c.y - sm.gy, uz = c.z - sm.gz;
                const double dc2 = ux * ux + uy * uy + uz * uz;
                if (sm.hl2 <= a.loc_eps2 * dc2) action = 4;
              }
            } else if (!cand) {
              if (cnt <= a.bucket) {
                action = 2;
                pfirst = fst;
                pcnt = cnt;
              } else {
                action = 3;
              }
            }
          }
        }
        if (LEARNED) {
          const unsigned cm = __ballot_sync(0xffffffffu, cand);
          if (cand) {
            const int q = (cqt + __popc(cm & lt)) & (kCandRing - 1);
            sm.cq_node[q] = node;
          }
          cqt += __popc(cm);
        }
      }
      // far-field entries
      const unsigned bm = __ballot_sync(0xffffffffu, action == 1);
      if (action == 1) sm.m2p[(m2t + __popc(bm & lt)) & (kM2pRing - 1)] = node;
      m2t += __popc(bm);
      // local-expansion entries
      const unsigned lm = __ballot_sync(0xffffffffu, action == 4);
      if (action == 4) sm.loc[(lct + __popc(lm & lt)) & (kLocRing - 1)] = node;
      lct += __popc(lm);
      // particle entries
      int ptot;
      const int pex = warp_excl_scan(action == 2 ? pcnt : 0, lane, &ptot);
      if (action == 2)
        for (int k = 0; k < pcnt; ++k)
          sm.p2p[(p2t + pex + k) & (kP2pRing - 1)] = pfirst + k;
      p2t += ptot;
      // opened twigs push their children (octant order)
      int4 k0 = make_int4(-1, -1, -1, -1), k1 = k0;
      if (action == 3) {
        const int4* kk = reinterpret_cast<const int4*>(a.kids + 8 * (int64_t)node);
        k0 = __ldg(kk);
        k1 = __ldg(kk + 1);
      }
      const int kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
      int kc = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) kc += kv[j] >= 0 ? 1 : 0;
      int ktot;
      const int kex = warp_excl_scan(kc, lane, &ktot);
      if (ssize + ktot > kStackCap) {
        overflow = true;
        break;
      }
      {
        int pos = ssize + kex;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (kv[j] >= 0) stack[pos++] = kv[j];
      }
      ssize += ktot;
      max_stack = max(max_stack, ssize);
      __syncwarp();
      while (p2t - p2h >= 32) {
        eval_p2p<PHYS, RDF>(sm, p2h, 32, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, tlx, tly,
                            tlz, close2, pt, tsp, act, lane, hist, acc);
        p2h += 32;
      }
      while (m2t - m2h >= 32) {
        if (RDF) eval_m2p_x2<ORDER>(sm, m2h, 32, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, lane, acc);
        else eval_m2p<ORDER>(sm, m2h, 32, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, lane, acc);
        m2h += 32;
      }
      while (lct - lch >= 32) {
        eval_local<ORDER>(sm, lch, 32, a, sm.gx, sm.gy, sm.gz, lane, lsum);
        lch += 32;
      }
    }
    if (overflow) {
      if (lane == 0) set_error(a.err, kErrWalk);
      continue;
    }
    if (p2t > p2h) {
      eval_p2p<PHYS, RDF>(sm, p2h, p2t - p2h, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, tlx,
                          tly, tlz, close2, pt, tsp, act, lane, hist, acc);
    }
    if (m2t > m2h) {
      if (RDF) eval_m2p_x2<ORDER>(sm, m2h, m2t - m2h, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, lane, acc);
      else eval_m2p<ORDER>(sm, m2h, m2t - m2h, a, sm.gx, sm.gy, sm.gz, thx, thy, thz, lane, acc);
    }
    if (lct > lch) {
      eval_local<ORDER>(sm, lch, lct - lch, a, sm.gx, sm.gy, sm.gz, lane, lsum);
    }
    if (lct > 0) {
      // every target evaluates the group's summed local expansion
      if (lane < kLocCoef) sm.loc_rows[lane] = lsum;
      __syncwarp();
      float lfx, lfy, lfz, lph, lpi;
      local_eval(sm.loc_rows, thx, thy, thz, lfx, lfy, lfz, lph, lpi);
      __syncwarp();
      kahan_add(acc.sx, acc.cx, lfx);
      kahan_add(acc.sy, acc.cy, lfy);
      kahan_add(acc.sz, acc.cz, lfz);
      phi_add(sm, lane, (double)lph, (double)lpi);
    }
    if (act) {
      const double sc = tsp ? kEps : -kEps;  // eps * target charge
      const int64_t o = a.order[pt];
      a.f[3 * o] = sc * ((double)acc.sx - (double)acc.cx);
      a.f[3 * o + 1] = sc * ((double)acc.sy - (double)acc.cy);
      a.f[3 * o + 2] = sc * ((double)acc.sz - (double)acc.cz);
      const double2 phi = sm.phi[lane];
      const double all = 0.5 * sc * phi.x;
      const double from_i = 0.5 * sc * phi.y;
      // Epot_e = ee + ie + ei, Epot_i = ii (tree.f90:674-715)
      a.epot_part[o] = tsp ? make_double2(all - from_i, from_i)
                           : make_double2(all, 0.0);
    }
    if (lane == 0) {
      // every queued entry was evaluated: the ring tails are the counts
      atomicAdd(&a.counters[0], (unsigned long long)m2t * n_act);
      atomicAdd(&a.counters[1], (unsigned long long)p2t * n_act);
      if (lct > 0) atomicAdd(&a.counters[8], (unsigned long long)lct);
    }
    if (LEARNED) {
      if (lane == 0) {
        atomicAdd(&a.counters[2], (unsigned long long)sm.n_mlp);
        atomicAdd(&a.counters[3], (unsigned long long)sm.n_fallback);
      }
    }
  }
  if (lane == 0) atomicMax(&a.control[1], max_stack);
  if (RDF) {
    // every warp of the block has left the group loop: add the block's bins
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * kRdfBins; i += blockDim.x) {
      const uint32_t v = hist[i];
      if (v) atomicAdd(&a.rdf[i], v);
    }
  }
}

// ------------------------------------------------------------- memory ----
template <class T>
static int realloc_dev(T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void**)p, count * sizeof(T)) == cudaSuccess ? 0 : 1;
}

int mixed_alloc_nodes(MixedBuffers& mb, int cap) {
  mb.cap = cap;
  int rc = 0;
  rc |= realloc_dev(&mb.kids, 8 * (size_t)cap);
  rc |= realloc_dev(&mb.first, (size_t)cap);
  rc |= realloc_dev(&mb.count, (size_t)cap);
  rc |= realloc_dev(&mb.digit, (size_t)cap);
  rc |= realloc_dev(&mb.m64, (size_t)kM64 * cap);
  rc |= realloc_dev(&mb.mom3, 3 * (size_t)cap);
  rc |= realloc_dev(&mb.mom4, 3 * (size_t)cap);
  rc |= realloc_dev(&mb.mom, 3 * (size_t)cap);
  rc |= realloc_dev(&mb.geom, (size_t)cap);
  rc |= realloc_dev(&mb.mac_k, (size_t)cap);
  rc |= realloc_dev(&mb.lvl_list, (size_t)cap);
  rc |= realloc_dev(&mb.cls, (size_t)net_cls_entries(cap));
  return rc;
}

int mixed_alloc_particles(MixedBuffers& mb, int n) {
  mb.n = n;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  mb.grid_warps = sms * kMaxBlocksPerSm * kMxWarps;
  int rc = 0;
  rc |= realloc_dev(&mb.xs, (size_t)n);
  rc |= realloc_dev(&mb.groups, (size_t)n);
  rc |= realloc_dev(&mb.stack, (size_t)mb.grid_warps * kStackCap);
  rc |= realloc_dev(&mb.control, 4);
  rc |= realloc_dev(&mb.lvl, 3 * (size_t)kLevelSlots);
  return rc;
}

void mixed_free(MixedBuffers& mb) {
  void* ptrs[] = {mb.kids, mb.first, mb.count, mb.digit, mb.m64, mb.mom,
                  mb.mom3, mb.mom4, mb.geom, mb.mac_k, mb.xs, mb.groups, mb.stack, mb.control,
                  mb.lvl_list, mb.lvl, mb.cls};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  mb = MixedBuffers();
}

MixedNodes mixed_nodes(const MixedBuffers& mb) {
  MixedNodes m;
  m.kids = mb.kids;
  m.first = mb.first;
  m.count = mb.count;
  m.digit = mb.digit;
  m.m64 = mb.m64;
  m.mom = mb.mom;
  m.mom3 = mb.mom3;
  m.mom4 = mb.mom4;
  m.geom = mb.geom;
  m.xs = mb.xs;
  m.groups = mb.groups;
  m.n_groups = mb.control + 2;
  m.lvl_list = mb.lvl_list;
  m.lvl = mb.lvl;
  m.cls = mb.cls;
  return m;
}

int walk_mixed(MixedBuffers& mb, const BuildBuffers& b, const double* x,
               int n, int n_el, const TreeView& tv, const WalkParams& wp,
               const MixedTuning& tune, const LearnedMac* learned,
               const Ensemble& ens, const float4* cloud_pk,
               double* f, double2* epot_part,
               uint32_t* rdf, unsigned long long* counters, int32_t* err,
               cudaStream_t st) {
  (void)x;
  if (n == 0) return 0;
  MixedArgs a;
  a.node_c = tv.node_c;
  a.mom = mb.mom;
  a.kids = mb.kids;
  a.first = mb.first;
  a.count = mb.count;
  a.xs = mb.xs;
  a.order = b.vals;
  a.bounds = tv.tree_bounds;
  a.groups = mb.groups;
  a.n_groups = mb.control + 2;
  a.n = n;
  a.n_el = n_el;
  a.control = mb.control;
  a.stack = mb.stack;
  a.bucket = tune.bucket < 1 ? 1 : (tune.bucket > kMaxBucket ? kMaxBucket : tune.bucket);
  // an accepted cell of at most p2p_max particles is summed as pairs: with
  // the hexadecapole far field (measured at N = 1M, learned criterion) one
  // far-field evaluation costs about two pair interactions, at order 3 about
  // four
  a.p2p_max = tune.order >= 4 ? 2 : (tune.order == 3 ? 4 : 2);
  if (a.p2p_max > a.bucket) a.p2p_max = a.bucket;
  a.loc_eps2 = (double)tune.loc_eps * tune.loc_eps;
  a.physics = wp.physics;
  a.inv_lam2_ee = (float)(1.0 / (wp.lam_ee * wp.lam_ee));
  a.inv_lam2_ei = (float)(1.0 / (wp.lam_ei * wp.lam_ei));
  a.inv_lam2_ii = (float)(1.0 / (wp.lam_ii * wp.lam_ii));
  a.inv_lam_ee = (float)(1.0 / wp.lam_ee);
  a.inv_lam_ei = (float)(1.0 / wp.lam_ei);
  a.inv_lam_ii = (float)(1.0 / wp.lam_ii);
  a.rs_inv = (float)(1.0 / wp.rs);
  a.dx_ei_inv_f = (float)(1.0 / wp.dx_ei);
  a.dx_ii_inv_f = (float)(1.0 / wp.dx_ii);
  a.f = f;
  a.epot_part = epot_part;
  a.rdf = rdf;
  a.counters = counters;
  a.err = err;
  // control[0] group cursor, [1] deepest stack; [2] (group count) is written
  // by the build
  cudaMemsetAsync(mb.control, 0, 2 * sizeof(int32_t), st);
  const bool L = learned != nullptr && learned->packed != nullptr &&
                 learned->f_prev != nullptr;
  a.packed = L ? learned->packed : nullptr;
  a.fmin = L ? learned->fmin : nullptr;
  a.fmax = L ? learned->fmax : nullptr;
  a.geom = mb.geom;
  a.mom3 = mb.mom3;
  a.mom4 = mb.mom4;
  a.margins = L ? learned->margins : nullptr;
  a.mac_k = mb.mac_k;
  a.f_prev = L ? learned->f_prev : nullptr;
  a.eta_over_eps = L ? (float)(learned->eta / kEps) : 0.f;
  a.rho_lo = L ? learned->rho_lo : 0.f;
  a.rho_hi = L ? learned->rho_hi : 0.f;
  a.lam_ei = (float)wp.lam_ei;
  a.nseg = ens.nseg;
  a.ens_start = ens.start;
  a.roots = ens.roots;
  a.cloud_pk = cloud_pk;
  int bps = tune.blocks_per_sm < 1 ? 1 : (tune.blocks_per_sm > kMaxBlocksPerSm ? kMaxBlocksPerSm : tune.blocks_per_sm);
  // the learned build holds at most kMinBlocksPerSmLearned blocks per SM:
  // more would only queue behind them
  if (L && bps > kMinBlocksPerSmLearned) bps = kMinBlocksPerSmLearned;
  const int sms_grid = mb.grid_warps / (kMaxBlocksPerSm * kMxWarps);
  int grid = sms_grid * bps;
  const bool r = rdf != nullptr;
  if (L) k_mac_node_terms<<<sms_grid * 4, 256, 0, st>>>(mb.geom, mb.mom3, tv.tree_bounds,
                                                       learned->margins, 1.f / learned->rho_hi,
                                                       mb.mac_k);
  int dev = 0;
  cudaGetDevice(&dev);
#define TG_LAUNCH(P, R, LL, O)                                                \
  do {                                                                        \
    auto kfn = k_walk_mixed<P, R, LL, O>;                                     \
    const size_t sb = walk_smem_bytes<LL, R>();                               \
    static unsigned attr_set = 0; /* devices with the smem limit raised */    \
    if (dev < 32 && !(attr_set & (1u << dev))) {                              \
      cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                           (int)sb);                                          \
      attr_set |= 1u << dev;                                                  \
    }                                                                         \
    kfn<<<R ? sms_grid : grid, R ? 32 * kRdfWarps : kMxThreads, sb, st>>>(a); \
  } while (0)
#define TG_LAUNCH_O(P, R, LL)                                                 \
  do {                                                                        \
    if (tune.order >= 4) TG_LAUNCH(P, R, LL, 4);                              \
    else if (tune.order == 3) TG_LAUNCH(P, R, LL, 3);                         \
    else TG_LAUNCH(P, R, LL, 2);                                              \
  } while (0)
  if (wp.physics == 1) {
    if (L) { if (r) TG_LAUNCH_O(1, true, true); else TG_LAUNCH_O(1, false, true); }
    else { if (r) TG_LAUNCH_O(1, true, false); else TG_LAUNCH_O(1, false, false); }
  } else {
    if (L) { if (r) TG_LAUNCH_O(0, true, true); else TG_LAUNCH_O(0, false, true); }
    else { if (r) TG_LAUNCH_O(0, true, false); else TG_LAUNCH_O(0, false, false); }
  }
#undef TG_LAUNCH_O
#undef TG_LAUNCH
  return L ? 2 : 1;
}

}  // namespace tg
