// mac_sample.cu -- training data for the learned MAC, generated on the GPU
// by the method itself.
//
// For every target group the kernel walks the combined tree with a fixed
// opening angle theta_g drawn per group from [theta_lo, theta_hi].  Every cell
// it tests whose acceptance ratio rho = s / (d - dx) lies in the band
// [rho_lo, rho_hi] becomes one sample: its 16 features (mac.cuh) and the
// exact error of accepting it for the group -- the FP64 multipole field at
// the walk's expansion order (net monopole + dipole + quadrupole, the
// octupole for order 3 and the hexadecapole for order 4, about the centroid)
// minus the FP64 Coulomb sum over
// the cell's particles, maximised over the group's targets.
// Cells with more than max_count particles are not sampled; the walk treats
// them with the fixed-theta test (they fall outside the training range).
// Each candidate is kept with probability `keep` (hash of cell and group) so
// that a bounded sample buffer spans many clouds.
#include "build.h"
#include "internal.cuh"
#include "mac.cuh"
#include "mlp.h"

namespace tg {

constexpr int kSmpWarps = 4;
constexpr int kSmpStack = 8192;

__device__ __forceinline__ float hash_unit(uint32_t a, uint32_t b) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u);
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return (h >> 8) * (1.f / 16777216.f);
}

__global__ void __launch_bounds__(32 * kSmpWarps)
    k_mac_sample(SampleArgs a) {
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * kSmpWarps + (threadIdx.x >> 5);
  int32_t* stack = a.stack + (int64_t)gwarp * kSmpStack;
  const unsigned lt = (1u << lane) - 1u;
  if (*((volatile int32_t*)a.err) & (kErrCapacity | kErrDepth | kErrNonFinite)) return;
  const int ngroups = *a.n_groups;
  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(a.cursor, 1);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= ngroups) break;
    const int2 grp = a.groups[g];
    const int p0 = grp.x, n_act = grp.y;
    const bool act = lane < n_act;
    const int pt = p0 + (act ? lane : n_act - 1);
    const double4 xt = a.xs[pt];
    double mn[3] = {xt.x, xt.y, xt.z}, mx[3] = {xt.x, xt.y, xt.z};
#pragma unroll
    for (int k = 0; k < 3; ++k)
      for (int o = 16; o > 0; o >>= 1) {
        mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
      }
    const double Gx = 0.5 * (mn[0] + mx[0]), Gy = 0.5 * (mn[1] + mx[1]), Gz = 0.5 * (mn[2] + mx[2]);
    const double hx = 0.5 * (mx[0] - mn[0]), hy = 0.5 * (mx[1] - mn[1]), hz = 0.5 * (mx[2] - mn[2]);
    const float hlen = (float)sqrt(hx * hx + hy * hy + hz * hz);
    const float theta_g = a.theta_lo + (a.theta_hi - a.theta_lo) * hash_unit((uint32_t)g, a.seed);
    int ssize = 1;
    if (lane == 0) stack[0] = 0;
    __syncwarp();
    while (ssize > 0) {
      const int nb = min(32, ssize);
      const int node = lane < nb ? stack[ssize - 1 - lane] : -1;
      ssize -= nb;
      __syncwarp();
      bool open = false, sample = false;
      double d = 0.0;
      if (node >= 0) {
        const double4 c = ldg_d4(&a.node_c[node]);
        if (c.w >= 0.0) {  // twig (leaves are summed directly by the walk)
          const float4 g4 = __ldg(&a.geom[node]);
          d = dist_to_box(c.x, c.y, c.z, Gx, Gy, Gz, hx, hy, hz);
          const double margin = d - (double)g4.y;
          const double rho = margin > 0.0 ? (double)g4.x / margin : 1e30;
          sample = rho >= a.rho_lo && rho <= a.rho_hi && g4.z <= (float)a.max_count &&
                   hash_unit((uint32_t)node * 2654435761u + (uint32_t)g, a.seed ^ 0x5bd1e995u) < a.keep;
          open = !(rho < (double)theta_g);
        }
      }
      // samples of this batch, one after the other
      unsigned sm = __ballot_sync(0xffffffffu, sample);
      while (sm) {
        const int L = __ffs(sm) - 1;
        sm &= sm - 1;
        const int cn = __shfl_sync(0xffffffffu, node, L);
        const double dd = __shfl_sync(0xffffffffu, d, L);
        int idx = 0;
        if (lane == L) idx = atomicAdd(a.n_out, 1);
        idx = __shfl_sync(0xffffffffu, idx, L);
        if (idx >= a.cap) continue;
        const double4 c = ldg_d4(&a.node_c[cn]);
        if (lane == L) {
          const float4 g4 = __ldg(&a.geom[cn]);
          const float4* mp = a.mom + 3 * (int64_t)cn;
          const float4* tp = a.mom3 + 3 * (int64_t)cn;
          mac_features(c.x, c.y, c.z, g4, __ldg(mp), __ldg(mp + 1), __ldg(mp + 2),
                       __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), Gx, Gy, Gz, hlen,
                       (float)dd, (float)n_act, a.feats + (int64_t)idx * kMacFeatures);
          a.extra[2 * (int64_t)idx] = (float)theta_g;
          a.extra[2 * (int64_t)idx + 1] = (float)(g4.x / (dd - g4.y));
        }
        // exact error of accepting cn for every target of the group (FP64)
        const double2* m = a.m64 + kM64 * (int64_t)cn;
        const double2 m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3], m4 = m[4], m5 = m[5];
        const double Q = m0.y, Dx = m1.x, Dy = m1.y, Dz = m2.x;
        const double Sxx = m3.x, Syy = m3.y, Szz = m4.x, Sxy = m4.y, Syz = m5.x, Szx = m5.y;
        const double ex = xt.x - c.x, ey = xt.y - c.y, ez = xt.z - c.z;
        const double r2 = ex * ex + ey * ey + ez * ez;
        const double ri = 1.0 / sqrt(r2);
        const double ri2 = ri * ri, ri3 = ri * ri2, ri5 = ri3 * ri2;
        const double Sx = Sxx * ex + Sxy * ey + Szx * ez;
        const double Sy = Sxy * ex + Syy * ey + Syz * ez;
        const double Sz = Szx * ex + Syz * ey + Szz * ez;
        const double u = ex * Sx + ey * Sy + ez * Sz;
        const double Dd = Dx * ex + Dy * ey + Dz * ez;
        const double gg = Q * ri3 + ri5 * (3.0 * Dd + 15.0 * u * ri2 - 3.0 * (Sxx + Syy + Szz));
        double fx = gg * ex - ri3 * Dx - 6.0 * ri5 * Sx;
        double fy = gg * ey - ri3 * Dy - 6.0 * ri5 * Sy;
        double fz = gg * ez - ri3 * Dz - 6.0 * ri5 * Sz;
        if (a.order >= 3) {  // octupole term, as in the walk (walk_mixed.cu)
          double T[10];
#pragma unroll
          for (int u2 = 0; u2 < 5; ++u2) {
            const double2 t2 = m[6 + u2];
            T[2 * u2] = t2.x;
            T[2 * u2 + 1] = t2.y;
          }
          const double xx = ex * ex, yy = ey * ey, zz = ez * ez;
          const double xy2 = 2 * ex * ey, xz2 = 2 * ex * ez, yz2 = 2 * ey * ez;
          const double Tx = T[0] * xx + T[5] * yy + T[7] * zz + T[3] * xy2 + T[4] * xz2 + T[9] * yz2;
          const double Ty = T[3] * xx + T[1] * yy + T[8] * zz + T[5] * xy2 + T[9] * xz2 + T[6] * yz2;
          const double Tz = T[4] * xx + T[6] * yy + T[2] * zz + T[9] * xy2 + T[7] * xz2 + T[8] * yz2;
          const double Vx = T[0] + T[5] + T[7], Vy = T[3] + T[1] + T[8], Vz = T[4] + T[6] + T[2];
          const double T3 = ex * Tx + ey * Ty + ez * Tz, Vd = Vx * ex + Vy * ey + Vz * ez;
          const double ri7 = ri5 * ri2;
          const double g3 = ri7 * (17.5 * ri2 * T3 - 7.5 * Vd);
          fx += g3 * ex - 7.5 * ri7 * Tx + 1.5 * ri5 * Vx;
          fy += g3 * ey - 7.5 * ri7 * Ty + 1.5 * ri5 * Vy;
          fz += g3 * ez - 7.5 * ri7 * Tz + 1.5 * ri5 * Vz;
        }
        if (a.order >= 4) {  // hexadecapole term, as in the walk (walk_mixed.cu)
          double H[16];
#pragma unroll
          for (int u2 = 0; u2 < 8; ++u2) {
            const double2 h2 = m[11 + u2];
            H[2 * u2] = h2.x;
            H[2 * u2 + 1] = h2.y;
          }
          // trace-free projection (order xxxx yyyy zzzz xxxy xxxz xyyy yyyz
          // xzzz yzzz xxyy xxzz yyzz xxyz xyyz xyzz)
          const double Cxx = H[0] + H[9] + H[10], Cyy = H[9] + H[1] + H[11],
                       Czz = H[10] + H[11] + H[2], Cxy = H[3] + H[5] + H[14],
                       Cxz = H[4] + H[13] + H[7], Cyz = H[12] + H[6] + H[8];
          const double tc = Cxx + Cyy + Czz, a7 = 1.0 / 7.0, a35 = 1.0 / 35.0;
          const double hxxxx = H[0] - 6.0 * a7 * Cxx + 3.0 * a35 * tc;
          const double hxxxy = H[3] - 3.0 * a7 * Cxy, hxxxz = H[4] - 3.0 * a7 * Cxz;
          const double hxxyy = H[9] - a7 * (Cxx + Cyy) + a35 * tc;
          const double hxxyz = H[12] - a7 * Cyz, hxyyy = H[5] - 3.0 * a7 * Cxy;
          const double hxyyz = H[13] - a7 * Cxz;
          const double hyyyy = H[1] - 6.0 * a7 * Cyy + 3.0 * a35 * tc;
          const double hyyyz = H[6] - 3.0 * a7 * Cyz;
          const double hxxzz = H[10] - a7 * (Cxx + Czz) + a35 * tc;
          const double hxyzz = H[14] - a7 * Cxy;
          const double hyyzz = H[11] - a7 * (Cyy + Czz) + a35 * tc;
          const double nx = ex * ri, ny = ey * ri, nz = ez * ri;
          const double xx = nx * nx, yy = ny * ny, zz = nz * nz;
          const double P1 = nx * (xx - 3.0 * zz), P2 = 3.0 * ny * (xx - zz);
          const double P3 = nz * (3.0 * xx - zz), P4 = 3.0 * nx * (yy - zz);
          const double P5 = 6.0 * nx * ny * nz, P6 = ny * (yy - 3.0 * zz);
          const double P7 = nz * (3.0 * yy - zz);
          const double Vx = hxxxx * P1 + hxxxy * P2 + hxxxz * P3 + hxxyy * P4 +
                            hxxyz * P5 + hxyyy * P6 + hxyyz * P7;
          const double Vy = hxxxy * P1 + hxxyy * P2 + hxxyz * P3 + hxyyy * P4 +
                            hxyyz * P5 + hyyyy * P6 + hyyyz * P7;
          const double Vz = hxxxz * P1 + hxxyz * P2 + hxxzz * P3 + hxyyz * P4 +
                            hxyzz * P5 + hyyyz * P6 + hyyzz * P7;
          const double H4 = nx * Vx + ny * Vy + nz * Vz;
          const double ri6 = ri3 * ri3;
          fx += 4.375 * ri6 * (9.0 * H4 * nx - 4.0 * Vx);
          fy += 4.375 * ri6 * (9.0 * H4 * ny - 4.0 * Vy);
          fz += 4.375 * ri6 * (9.0 * H4 * nz - 4.0 * Vz);
        }
        const int j0 = __ldg(&a.first[cn]), j1 = j0 + __ldg(&a.count[cn]);
        for (int j = j0; j < j1; ++j) {
          const double4 s = a.xs[j];
          if (j == pt) continue;
          const double qx = xt.x - s.x, qy = xt.y - s.y, qz = xt.z - s.z;
          const double q2 = qx * qx + qy * qy + qz * qz;
          if (q2 == 0.0) continue;
          const double qi = 1.0 / sqrt(q2);
          const double w = (s.w > 0.5 ? 1.0 : -1.0) * qi * qi * qi;
          fx -= w * qx;
          fy -= w * qy;
          fz -= w * qz;
        }
        double err = act ? sqrt(fx * fx + fy * fy + fz * fz) : 0.0;
        for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if (lane == 0) {
          const double scale = (double)__ldg(&a.geom[cn]).z / (dd * dd);
          a.labels[idx] = (float)log10(fmax(err / scale, 1e-12));
        }
      }
      // traversal continues with the fixed theta_g decision
      int4 k0 = make_int4(-1, -1, -1, -1), k1 = k0;
      if (open) {
        const int4* kk = reinterpret_cast<const int4*>(a.kids + 8 * (int64_t)node);
        k0 = __ldg(kk);
        k1 = __ldg(kk + 1);
      }
      const int kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
      int kc = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) kc += kv[j] >= 0 ? 1 : 0;
      int inc = kc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      const int ktot = __shfl_sync(0xffffffffu, inc, 31);
      if (ssize + ktot > kSmpStack) {
        if (lane == 0) set_error(a.err, kErrWalk);
        break;
      }
      int pos = ssize + inc - kc;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (kv[j] >= 0) stack[pos++] = kv[j];
      ssize += ktot;
      __syncwarp();
      (void)lt;
    }
  }
}

int mac_sample(const SampleArgs& a, int grid_warps, cudaStream_t st) {
  cudaMemsetAsync(a.cursor, 0, sizeof(int32_t), st);
  int blocks = grid_warps / kSmpWarps;
  k_mac_sample<<<blocks, 32 * kSmpWarps, 0, st>>>(a);
  return 1;
}

int mac_sample_stack_per_warp() { return kSmpStack; }

}  // namespace tg
