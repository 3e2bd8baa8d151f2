// local.cuh -- second-order local (Taylor) expansion of a far cell's field
// about the centre of a target group.
//
// A cell far from a group (group half-diagonal h small against the distance
// d0 from the group centre G to the cell's centroid) has nearly the same
// field at every target of the group.  Instead of 32 lanes each evaluating
// the cell's multipole series at their own target (the M2P of the walk), one
// lane expands the cell's potential phi about G:
//   phi(G + t) = phi0 + g.t + 1/2 t.H.t + 1/6 K(t,t,t) + 1/24 L(t,t,t,t) + O(|t|^5)
// with g = grad phi, H = grad grad phi, K = grad^3 phi, L = grad^4 phi at G,
// and the warp
// sums the coefficients of all such cells; every target then evaluates the
// summed expansion once at its own offset t.  The force -grad phi is kept to
// third order in t, so its truncation error relative to the cell's field is
// of order (h/d0)^4.
//
// Multipole convention (the walk's, about the centroid, d = target -
// centroid, r = |d|):
//   phi = Q/r + D.d/r^3 + 3 d.S.d/r^5 + 5/2 T(d,d,d)/r^7 + 35/8 H(d,d,d,d)/r^9
// with S, T, H trace-free.  Equivalently phi = Q G - D_i G_i + S_ij G_ij -
// 1/6 T_ijk G_ijk + 1/24 H_ijkl G_ijkl, G_{i..} the derivatives of 1/r.
// phi0, g and H carry every order the walk uses, K the multipoles to T, L
// those to S (each dropped term is smaller than a kept one by a further
// factor a/d0 or h/d0).  All of it is in normalised form
// (unit vector n = d/r, s = 1/r, each moment scaled by its power of s first)
// so that cells and groups millions of um apart stay finite in FP32.
//
// Coefficient layout (kLocCoef floats):
//   0 phi0 | 1..3 g | 4..8 Hxx Hyy Hxy Hxz Hyz (Hzz = -Hxx - Hyy) |
//   9..15 Kxxx Kyyy Kxxy Kxxz Kxyy Kyyz Kxyz (the rest from the traces) |
//   16 phi_ion0 (q_ion / r) | 17..19 grad (q_ion / r) |
//   20..28 Lxxxx Lxxxy Lxxyy Lxyyy Lyyyy Lxxxz Lxxyz Lxyyz Lyyyz (the rest
//   from the traces)
// H, K and L are trace-free because every multipole term is harmonic.
#pragma once

#ifdef __CUDACC__
#define TG_LOC_HD __host__ __device__ __forceinline__
#define TG_LOC_RSQRT(x) rsqrtf(x)
#else
#include <cmath>
#define TG_LOC_HD inline
#define TG_LOC_RSQRT(x) (1.f / std::sqrt(x))
#endif

namespace tg {

constexpr int kLocCoef = 29;

// FP32 moments of one cell about its centroid, in the walk's storage order.
struct CellMoments {
  float q;       // net charge
  float d[3];    // dipole
  float s[6];    // trace-free 1/2 sum q a a: xx yy zz xy yz zx
  float t[10];   // trace-free sum q a a a: xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
  float h[12];   // trace-free sum q a a a a: xxxx xxxy xxxz xxyy xxyz xyyy
                 // xyyz yyyy yyyz xxzz xyzz yyzz
  float q_ion;   // ion count (the Epot_e / Epot_i split, monopole order)
};

// The fourth-derivative tensor of the net charge, dipole and second-moment
// terms: its component (M, P, Q, R) from the unit vector n and the scalar,
// vector and matrix coefficients of each index structure (all indices are
// compile-time, so the Kronecker deltas fold away).
struct LocalL4 {
  float a4, b4, c4, s210, sm30;
  float n[3], v[3], w[3];
  float S[3][3];
  // one (pair | rest) split of the four indices: S_ab n_c n_d, d_ab n_c n_d,
  // S_ab d_cd and (n_a w_b + n_b w_a) d_cd
  template <int A, int B, int C, int D>
  TG_LOC_HD float split() const {
    float t = s210 * S[A][B] * n[C] * n[D];
    if (A == B) t = fmaf(b4, n[C] * n[D], t);
    if (C == D) t += fmaf(sm30, S[A][B], fmaf(n[A], w[B], n[B] * w[A]));
    return t;
  }
  template <int M, int P, int Q, int R>
  TG_LOC_HD float comp() const {
    float t = a4 * n[M] * n[P] * n[Q] * n[R];
    t = fmaf(v[M], n[P] * n[Q] * n[R], t);
    t = fmaf(v[P], n[M] * n[Q] * n[R], t);
    t = fmaf(v[Q], n[M] * n[P] * n[R], t);
    t = fmaf(v[R], n[M] * n[P] * n[Q], t);
    t += split<M, P, Q, R>() + split<Q, R, M, P>() + split<M, Q, P, R>() +
         split<P, R, M, Q>() + split<M, R, P, Q>() + split<P, Q, M, R>();
    constexpr int pairs = (M == P && Q == R) + (M == Q && P == R) + (M == R && P == Q);
    if (pairs) t = fmaf((float)pairs, c4, t);
    return t;
  }
};

// Coefficients of one cell's expansion about the group centre; (dx, dy, dz)
// = G - centroid.  ORDER (2..4) is the far-field order of phi0 and g.
template <int ORDER>
TG_LOC_HD void local_coefs(float dx, float dy, float dz, const CellMoments& m, float* c) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 1e-30f)));
  const float s = TG_LOC_RSQRT(r2), s2 = s * s;
  const float nx = dx * s, ny = dy * s, nz = dz * s;
  const float Q = m.q, Dx = m.d[0], Dy = m.d[1], Dz = m.d[2];
  const float Sxx = m.s[0], Syy = m.s[1], Szz = m.s[2], Sxy = m.s[3], Syz = m.s[4],
              Szx = m.s[5];
  // S n, n.S.n, D.n
  const float Snx = fmaf(Sxx, nx, fmaf(Sxy, ny, Szx * nz));
  const float Sny = fmaf(Sxy, nx, fmaf(Syy, ny, Syz * nz));
  const float Snz = fmaf(Szx, nx, fmaf(Syz, ny, Szz * nz));
  const float u = fmaf(nx, Snx, fmaf(ny, Sny, nz * Snz));
  const float Dn = fmaf(Dx, nx, fmaf(Dy, ny, Dz * nz));
  // T(., n, n), T(n, n, n) and the matrix T(., ., n)
  float Tx = 0.f, Ty = 0.f, Tz = 0.f, T3 = 0.f;
  float TNxx = 0.f, TNyy = 0.f, TNxy = 0.f, TNxz = 0.f, TNyz = 0.f;
  if (ORDER >= 3) {
    const float Txxx = m.t[0], Tyyy = m.t[1], Txxy = m.t[3], Txxz = m.t[4],
                Txyy = m.t[5], Tyyz = m.t[6], Txzz = m.t[7], Tyzz = m.t[8], Txyz = m.t[9];
    const float zz = nz * nz;
    const float a2 = fmaf(nx, nx, -zz), b2 = fmaf(ny, ny, -zz);
    const float xy2 = 2.f * nx * ny, xz2 = 2.f * nx * nz, yz2 = 2.f * ny * nz;
    Tx = fmaf(Txxx, a2, fmaf(Txyy, b2, fmaf(Txxy, xy2, fmaf(Txxz, xz2, Txyz * yz2))));
    Ty = fmaf(Txxy, a2, fmaf(Tyyy, b2, fmaf(Txyy, xy2, fmaf(Txyz, xz2, Tyyz * yz2))));
    Tz = fmaf(Txxz, a2, fmaf(Tyyz, b2, fmaf(Txyz, xy2, fmaf(Txzz, xz2, Tyzz * yz2))));
    T3 = fmaf(nx, Tx, fmaf(ny, Ty, nz * Tz));
    TNxx = fmaf(Txxx, nx, fmaf(Txxy, ny, Txxz * nz));
    TNyy = fmaf(Txyy, nx, fmaf(Tyyy, ny, Tyyz * nz));
    TNxy = fmaf(Txxy, nx, fmaf(Txyy, ny, Txyz * nz));
    TNxz = fmaf(Txxz, nx, fmaf(Txyz, ny, Txzz * nz));
    TNyz = fmaf(Txyz, nx, fmaf(Tyyz, ny, Tyzz * nz));
  }
  // H(., n, n, n) through the cubic harmonics P1..P7 of n, H(n, n, n, n)
  float Vx = 0.f, Vy = 0.f, Vz = 0.f, H4 = 0.f;
  if (ORDER >= 4) {
    const float* H = m.h;
    const float xx = nx * nx, yy = ny * ny, zz3 = 3.f * nz * nz;
    const float P1 = nx * (xx - zz3);
    const float P6 = ny * (yy - zz3);
    const float P2 = 3.f * ny * fmaf(nz, -nz, xx);
    const float P4 = 3.f * nx * fmaf(nz, -nz, yy);
    const float P3 = nz * fmaf(3.f, xx, -nz * nz);
    const float P7 = nz * fmaf(3.f, yy, -nz * nz);
    const float P5 = 6.f * nx * ny * nz;
    Vx = fmaf(H[0], P1, fmaf(H[1], P2, fmaf(H[2], P3, fmaf(H[3], P4,
         fmaf(H[4], P5, fmaf(H[5], P6, H[6] * P7))))));
    Vy = fmaf(H[1], P1, fmaf(H[3], P2, fmaf(H[4], P3, fmaf(H[5], P4,
         fmaf(H[6], P5, fmaf(H[7], P6, H[8] * P7))))));
    Vz = fmaf(H[2], P1, fmaf(H[4], P2, fmaf(H[9], P3, fmaf(H[6], P4,
         fmaf(H[10], P5, fmaf(H[8], P6, H[11] * P7))))));
    H4 = fmaf(nx, Vx, fmaf(ny, Vy, nz * Vz));
  }
  // phi0 and g = grad phi at G: r phi = php, r^2 (-grad phi) = gp n + gv
  const float gp = fmaf(s, fmaf(s, fmaf(s, fmaf(39.375f * s, H4, 17.5f * T3), 15.f * u), 3.f * Dn), Q);
  const float php = fmaf(s, fmaf(s, fmaf(s, fmaf(4.375f * s, H4, 2.5f * T3), 3.f * u), Dn), Q);
  const float c5 = -6.f * s2, c7 = -7.5f * s2 * s, c9 = -17.5f * s2 * s2;
  const float gvx = fmaf(c9, Vx, fmaf(c7, Tx, fmaf(c5, Snx, -s * Dx)));
  const float gvy = fmaf(c9, Vy, fmaf(c7, Ty, fmaf(c5, Sny, -s * Dy)));
  const float gvz = fmaf(c9, Vz, fmaf(c7, Tz, fmaf(c5, Snz, -s * Dz)));
  c[0] = s * php;
  c[1] = -s2 * fmaf(gp, nx, gvx);
  c[2] = -s2 * fmaf(gp, ny, gvy);
  c[3] = -s2 * fmaf(gp, nz, gvz);
  // H = s^3 [al n n + be I + n w + w n + s^2 (6 S + 15 s T(., ., n)
  //      + 52.5 s^2 H(., ., n, n))], every multipole order of the walk
  const float s3 = s2 * s;
  const float al = fmaf(s, fmaf(s, fmaf(s, fmaf(433.125f * s, H4, 157.5f * T3), 105.f * u),
                                15.f * Dn), 3.f * Q);
  const float be = -fmaf(s, fmaf(s, fmaf(s, fmaf(39.375f * s, H4, 17.5f * T3), 15.f * u),
                                 3.f * Dn), Q);
  const float wx = -s * fmaf(s, fmaf(s, fmaf(157.5f * s, Vx, 52.5f * Tx), 30.f * Snx), 3.f * Dx);
  const float wy = -s * fmaf(s, fmaf(s, fmaf(157.5f * s, Vy, 52.5f * Ty), 30.f * Sny), 3.f * Dy);
  const float wz = -s * fmaf(s, fmaf(s, fmaf(157.5f * s, Vz, 52.5f * Tz), 30.f * Snz), 3.f * Dz);
  // H(., ., n, n)
  float HNxx = 0.f, HNyy = 0.f, HNxy = 0.f, HNxz = 0.f, HNyz = 0.f;
  if (ORDER >= 4) {
    const float* H = m.h;
    const float xx = nx * nx, yy = ny * ny, zz = nz * nz;
    const float xy2 = 2.f * nx * ny, xz2 = 2.f * nx * nz, yz2 = 2.f * ny * nz;
    const float Hxzzz = -(H[2] + H[6]), Hyzzz = -(H[4] + H[8]);
    HNxx = fmaf(H[0], xx, fmaf(H[3], yy, fmaf(H[9], zz, fmaf(H[1], xy2, fmaf(H[2], xz2, H[4] * yz2)))));
    HNyy = fmaf(H[3], xx, fmaf(H[7], yy, fmaf(H[11], zz, fmaf(H[5], xy2, fmaf(H[6], xz2, H[8] * yz2)))));
    HNxy = fmaf(H[1], xx, fmaf(H[5], yy, fmaf(H[10], zz, fmaf(H[3], xy2, fmaf(H[4], xz2, H[6] * yz2)))));
    HNxz = fmaf(H[2], xx, fmaf(H[6], yy, fmaf(Hxzzz, zz, fmaf(H[4], xy2, fmaf(H[9], xz2, H[10] * yz2)))));
    HNyz = fmaf(H[4], xx, fmaf(H[8], yy, fmaf(Hyzzz, zz, fmaf(H[6], xy2, fmaf(H[10], xz2, H[11] * yz2)))));
  }
  const float s15 = 15.f * s, s525 = 52.5f * s2;
  // the traceless-moment part s^2 (6 S + 15 s TN + 52.5 s^2 HN) per component
  const float Mxx = s2 * fmaf(s525, HNxx, fmaf(s15, TNxx, 6.f * Sxx));
  const float Myy = s2 * fmaf(s525, HNyy, fmaf(s15, TNyy, 6.f * Syy));
  const float Mxy = s2 * fmaf(s525, HNxy, fmaf(s15, TNxy, 6.f * Sxy));
  const float Mxz = s2 * fmaf(s525, HNxz, fmaf(s15, TNxz, 6.f * Szx));
  const float Myz = s2 * fmaf(s525, HNyz, fmaf(s15, TNyz, 6.f * Syz));
  c[4] = s3 * fmaf(al * nx, nx, fmaf(2.f * nx, wx, Mxx + be));
  c[5] = s3 * fmaf(al * ny, ny, fmaf(2.f * ny, wy, Myy + be));
  c[6] = s3 * fmaf(al * nx, ny, fmaf(nx, wy, fmaf(ny, wx, Mxy)));
  c[7] = s3 * fmaf(al * nx, nz, fmaf(nx, wz, fmaf(nz, wx, Mxz)));
  c[8] = s3 * fmaf(al * ny, nz, fmaf(ny, wz, fmaf(nz, wy, Myz)));
  // K = -s^4 [A nnn + B (n d)_3 + (V n n)_3 + (W d)_3 + s^2 (30 (S n)_3
  //      + s (105 (T(., ., n) n)_3 - 15 T))], ( )_3 the three index
  // placements; multipoles to T
  const float A = fmaf(s, fmaf(s, fmaf(1732.5f * s, T3, 945.f * u), 105.f * Dn), 15.f * Q);
  const float B = -fmaf(s, fmaf(s, fmaf(157.5f * s, T3, 105.f * u), 15.f * Dn), 3.f * Q);
  const float Vkx = -s * fmaf(s, fmaf(472.5f * s, Tx, 210.f * Snx), 15.f * Dx);
  const float Vky = -s * fmaf(s, fmaf(472.5f * s, Ty, 210.f * Sny), 15.f * Dy);
  const float Vkz = -s * fmaf(s, fmaf(472.5f * s, Tz, 210.f * Snz), 15.f * Dz);
  const float Wx = s * fmaf(s, fmaf(52.5f * s, Tx, 30.f * Snx), 3.f * Dx);
  const float Wy = s * fmaf(s, fmaf(52.5f * s, Ty, 30.f * Sny), 3.f * Dy);
  const float Wz = s * fmaf(s, fmaf(52.5f * s, Tz, 30.f * Snz), 3.f * Dz);
  const float ms4 = -s2 * s2, s105 = 105.f * s, m15s = -15.f * s;
  const float xx = nx * nx, yy = ny * ny;
  // the moment part s^2 (30 Sc + s (105 TNc - 15 Tc)) of one component
  auto km = [&](float Sc, float TNc, float Tc) {
    return s2 * fmaf(s105, TNc, fmaf(m15s, Tc, 30.f * Sc));
  };
  // T itself (not read below order 3)
  const float Txxx = ORDER >= 3 ? m.t[0] : 0.f, Tyyy = ORDER >= 3 ? m.t[1] : 0.f,
              Txxy = ORDER >= 3 ? m.t[3] : 0.f, Txxz = ORDER >= 3 ? m.t[4] : 0.f,
              Txyy = ORDER >= 3 ? m.t[5] : 0.f, Tyyz = ORDER >= 3 ? m.t[6] : 0.f,
              Txyz = ORDER >= 3 ? m.t[9] : 0.f;
  // K_mmm = A n_m^3 + 3 B n_m + 3 V_m n_m^2 + 3 W_m + moments
  c[9] = ms4 * fmaf(A * xx, nx, fmaf(3.f, fmaf(B, nx, fmaf(Vkx * nx, nx, Wx)),
                                     km(3.f * Sxx * nx, 3.f * TNxx * nx, Txxx)));
  c[10] = ms4 * fmaf(A * yy, ny, fmaf(3.f, fmaf(B, ny, fmaf(Vky * ny, ny, Wy)),
                                      km(3.f * Syy * ny, 3.f * TNyy * ny, Tyyy)));
  // K_mmq (m != q) = A n_m^2 n_q + B n_q + 2 V_m n_m n_q + V_q n_m^2 + W_q + moments
  c[11] = ms4 * fmaf(A * xx, ny, fmaf(B, ny, fmaf(2.f * Vkx * nx, ny, fmaf(Vky, xx, Wy +
              km(fmaf(2.f * Sxy, nx, Sxx * ny), fmaf(2.f * TNxy, nx, TNxx * ny), Txxy)))));
  c[12] = ms4 * fmaf(A * xx, nz, fmaf(B, nz, fmaf(2.f * Vkx * nx, nz, fmaf(Vkz, xx, Wz +
              km(fmaf(2.f * Szx, nx, Sxx * nz), fmaf(2.f * TNxz, nx, TNxx * nz), Txxz)))));
  c[13] = ms4 * fmaf(A * yy, nx, fmaf(B, nx, fmaf(2.f * Vky * ny, nx, fmaf(Vkx, yy, Wx +
              km(fmaf(2.f * Sxy, ny, Syy * nx), fmaf(2.f * TNxy, ny, TNyy * nx), Txyy)))));
  c[14] = ms4 * fmaf(A * yy, nz, fmaf(B, nz, fmaf(2.f * Vky * ny, nz, fmaf(Vkz, yy, Wz +
              km(fmaf(2.f * Syz, ny, Syy * nz), fmaf(2.f * TNyz, ny, TNyy * nz), Tyyz)))));
  // K_xyz = A nx ny nz + Vx ny nz + Vy nx nz + Vz nx ny + moments
  c[15] = ms4 * fmaf(A * nx * ny, nz, fmaf(Vkx, ny * nz, fmaf(Vky, nx * nz, fmaf(Vkz, nx * ny,
              km(fmaf(Syz, nx, fmaf(Szx, ny, Sxy * nz)),
                 fmaf(TNxy, nz, fmaf(TNxz, ny, TNyz * nx)), Txyz)))));
  // ion monopole for the Epot split
  const float qs = m.q_ion * s;
  c[16] = qs;
  c[17] = -qs * s * nx;
  c[18] = -qs * s * ny;
  c[19] = -qs * s * nz;
  // L = grad^4 phi, multipoles to S:
  //   s^5 [a4 nnnn + b4 (d n n)_6 + c4 (d d)_3 + (V4 n n n)_4 + (n W4 d)_12
  //        + 210 s^2 (S n n)_6 - 30 s^2 (S d)_6]
  LocalL4 l;
  l.a4 = fmaf(s, fmaf(10395.f * s, u, 945.f * Dn), 105.f * Q);
  l.b4 = -fmaf(s, fmaf(945.f * s, u, 105.f * Dn), 15.f * Q);
  l.c4 = fmaf(s, fmaf(105.f * s, u, 15.f * Dn), 3.f * Q);
  l.n[0] = nx; l.n[1] = ny; l.n[2] = nz;
  l.v[0] = -s * fmaf(1890.f * s, Snx, 105.f * Dx);
  l.v[1] = -s * fmaf(1890.f * s, Sny, 105.f * Dy);
  l.v[2] = -s * fmaf(1890.f * s, Snz, 105.f * Dz);
  l.w[0] = s * fmaf(210.f * s, Snx, 15.f * Dx);
  l.w[1] = s * fmaf(210.f * s, Sny, 15.f * Dy);
  l.w[2] = s * fmaf(210.f * s, Snz, 15.f * Dz);
  l.S[0][0] = Sxx; l.S[1][1] = Syy; l.S[2][2] = Szz;
  l.S[0][1] = l.S[1][0] = Sxy; l.S[1][2] = l.S[2][1] = Syz; l.S[0][2] = l.S[2][0] = Szx;
  l.s210 = 210.f * s2;
  l.sm30 = -30.f * s2;
  const float s5 = s3 * s2;
  c[20] = s5 * l.comp<0, 0, 0, 0>();
  c[21] = s5 * l.comp<0, 0, 0, 1>();
  c[22] = s5 * l.comp<0, 0, 1, 1>();
  c[23] = s5 * l.comp<0, 1, 1, 1>();
  c[24] = s5 * l.comp<1, 1, 1, 1>();
  c[25] = s5 * l.comp<0, 0, 0, 2>();
  c[26] = s5 * l.comp<0, 0, 1, 2>();
  c[27] = s5 * l.comp<0, 1, 1, 2>();
  c[28] = s5 * l.comp<1, 1, 1, 2>();
}

// Evaluates summed coefficients at the offset t from the group centre:
// force f = -grad phi (unscaled), potential phi and its ion part.
TG_LOC_HD void local_eval(const float* c, float tx, float ty, float tz, float& fx,
                          float& fy, float& fz, float& phi, float& phi_ion) {
  const float Hxx = c[4], Hyy = c[5], Hxy = c[6], Hxz = c[7], Hyz = c[8];
  const float Hzz = -(Hxx + Hyy);
  const float Kxxx = c[9], Kyyy = c[10], Kxxy = c[11], Kxxz = c[12], Kxyy = c[13],
              Kyyz = c[14], Kxyz = c[15];
  const float Kxzz = -(Kxxx + Kxyy), Kyzz = -(Kxxy + Kyyy), Kzzz = -(Kxxz + Kyyz);
  const float Htx = fmaf(Hxx, tx, fmaf(Hxy, ty, Hxz * tz));
  const float Hty = fmaf(Hxy, tx, fmaf(Hyy, ty, Hyz * tz));
  const float Htz = fmaf(Hxz, tx, fmaf(Hyz, ty, Hzz * tz));
  const float xx = tx * tx, yy = ty * ty, zz = tz * tz;
  const float xy2 = 2.f * tx * ty, xz2 = 2.f * tx * tz, yz2 = 2.f * ty * tz;
  const float Kx = fmaf(Kxxx, xx, fmaf(Kxyy, yy, fmaf(Kxzz, zz, fmaf(Kxxy, xy2, fmaf(Kxxz, xz2, Kxyz * yz2)))));
  const float Ky = fmaf(Kxxy, xx, fmaf(Kyyy, yy, fmaf(Kyzz, zz, fmaf(Kxyy, xy2, fmaf(Kxyz, xz2, Kyyz * yz2)))));
  const float Kz = fmaf(Kxxz, xx, fmaf(Kyyz, yy, fmaf(Kzzz, zz, fmaf(Kxyz, xy2, fmaf(Kxzz, xz2, Kyzz * yz2)))));
  // L(t, t, t, .) from the nine stored components (xxxx xxxy xxyy xyyy yyyy
  // xxxz xxyz xyyz yyyz) and the traces
  const float* L = c + 20;
  const float Lxxzz = -(L[0] + L[2]), Lxyzz = -(L[1] + L[3]), Lyyzz = -(L[2] + L[4]);
  const float Lxzzz = -(L[5] + L[7]), Lyzzz = -(L[6] + L[8]), Lzzzz = -(Lxxzz + Lyyzz);
  const float x3 = xx * tx, y3 = yy * ty, z3 = zz * tz;
  const float x2y = 3.f * xx * ty, x2z = 3.f * xx * tz, xy2b = 3.f * tx * yy;
  const float y2z = 3.f * yy * tz, xz2b = 3.f * tx * zz, yz2b = 3.f * ty * zz;
  const float xyz = 6.f * tx * ty * tz;
  const float Lx = fmaf(L[0], x3, fmaf(L[1], x2y, fmaf(L[5], x2z, fmaf(L[2], xy2b, fmaf(L[6], xyz,
                   fmaf(Lxxzz, xz2b, fmaf(L[3], y3, fmaf(L[7], y2z, fmaf(Lxyzz, yz2b, Lxzzz * z3)))))))));
  const float Ly = fmaf(L[1], x3, fmaf(L[2], x2y, fmaf(L[6], x2z, fmaf(L[3], xy2b, fmaf(L[7], xyz,
                   fmaf(Lxyzz, xz2b, fmaf(L[4], y3, fmaf(L[8], y2z, fmaf(Lyyzz, yz2b, Lyzzz * z3)))))))));
  const float Lz = fmaf(L[5], x3, fmaf(L[6], x2y, fmaf(Lxxzz, x2z, fmaf(L[7], xy2b, fmaf(Lxyzz, xyz,
                   fmaf(Lxzzz, xz2b, fmaf(L[8], y3, fmaf(Lyyzz, y2z, fmaf(Lyzzz, yz2b, Lzzzz * z3)))))))));
  // grad phi(t) = g + H t + 1/2 K(t, t, .) + 1/6 L(t, t, t, .)
  const float sixth = 1.f / 6.f;
  const float gx = fmaf(sixth, Lx, fmaf(0.5f, Kx, c[1] + Htx));
  const float gy = fmaf(sixth, Ly, fmaf(0.5f, Ky, c[2] + Hty));
  const float gz = fmaf(sixth, Lz, fmaf(0.5f, Kz, c[3] + Htz));
  fx = -gx;
  fy = -gy;
  fz = -gz;
  // phi(t) = phi0 + g.t + 1/2 t.H.t + 1/6 K(t, t, t) + 1/24 L(t, t, t, t)
  const float tHt = fmaf(tx, Htx, fmaf(ty, Hty, tz * Htz));
  const float tKt = fmaf(tx, Kx, fmaf(ty, Ky, tz * Kz));
  const float tLt = fmaf(tx, Lx, fmaf(ty, Ly, tz * Lz));
  phi = c[0] + fmaf(c[1], tx, fmaf(c[2], ty, fmaf(c[3], tz,
               fmaf(0.5f, tHt, fmaf(sixth, tKt, tLt * (1.f / 24.f))))));
  phi_ion = c[16] + fmaf(c[17], tx, fmaf(c[18], ty, c[19] * tz));
}

}  // namespace tg
