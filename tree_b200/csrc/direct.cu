// direct.cu -- FP64 O(N^2) direct sum over every source for a list of targets
// (compiled -fmad=false).  This is the accuracy judge of the tree paths: the
// theta -> 0 limit of the walk, with the same leaf pair laws.
//
// Grid: x = tiles of 128 targets, y = contiguous chunks of sources.  Each
// block stages its sources through shared memory and writes one partial
// (fx, fy, fz, 0.5 V) per target and chunk; k_direct_reduce sums the chunks
// in fixed order, so results do not depend on scheduling.
#include "direct.h"
#include "internal.cuh"
#include "pair64.cuh"

namespace tg {

constexpr int kDirT = 128;

template <int PHYS>
__global__ void __launch_bounds__(kDirT)
    k_direct(const double* __restrict__ x, int n, int n_el,
             const int64_t* __restrict__ targets, int nt, int chunk,
             WalkParams wp, double4* __restrict__ partial) {
  __shared__ double4 src[kDirT];
  int t = blockIdx.x * kDirT + threadIdx.x;
  bool active = t < nt;
  int64_t o = active ? targets[t] : 0;
  int tsp = o >= n_el;
  double xt0 = 0, xt1 = 0, xt2 = 0;
  if (active) {
    xt0 = x[3 * o];
    xt1 = x[3 * o + 1];
    xt2 = x[3 * o + 2];
  }
  double f0 = 0.0, f1 = 0.0, f2 = 0.0, ep = 0.0;
  int j0 = blockIdx.y * chunk;
  int j1 = j0 + chunk < n ? j0 + chunk : n;
  for (int base = j0; base < j1; base += kDirT) {
    int j = base + threadIdx.x;
    if (j < j1)
      src[threadIdx.x] = make_double4(x[3 * (int64_t)j], x[3 * (int64_t)j + 1],
                                      x[3 * (int64_t)j + 2], (double)j);
    __syncthreads();
    int m = j1 - base < kDirT ? j1 - base : kDirT;
    if (active) {
      for (int k = 0; k < m; ++k) {
        double4 s = src[k];
        int js = (int)s.w;
        bool same = (js >= n_el) == (tsp == 1);
        double xr0 = xt0 - s.x, xr1 = xt1 - s.y, xr2 = xt2 - s.z;
        double r2 = xr0 * xr0 + xr1 * xr1 + xr2 * xr2;
        double r;
        leaf_pair64<PHYS>(xr0, xr1, xr2, r2, same, tsp, js == (int)o, wp, f0,
                          f1, f2, ep, r);
      }
    }
    __syncthreads();
  }
  if (active) partial[(int64_t)blockIdx.y * nt + t] = make_double4(f0, f1, f2, ep);
}

__global__ void k_direct_reduce(const double4* __restrict__ partial, int nt,
                                int nchunks, double* __restrict__ f,
                                double* __restrict__ epot) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double f0 = 0, f1 = 0, f2 = 0, ep = 0;
  for (int c = 0; c < nchunks; ++c) {
    double4 p = partial[(int64_t)c * nt + t];
    f0 += p.x;
    f1 += p.y;
    f2 += p.z;
    ep += p.w;
  }
  f[3 * (int64_t)t] = f0;
  f[3 * (int64_t)t + 1] = f1;
  f[3 * (int64_t)t + 2] = f2;
  epot[t] = ep;
}

int direct_chunks(int n, int nt) {
  // enough blocks to fill 148 SMs several times over
  int tiles = (nt + kDirT - 1) / kDirT;
  int want = (8 * 148 + tiles - 1) / (tiles > 0 ? tiles : 1);
  int maxc = (n + kDirT - 1) / kDirT;
  if (want > maxc) want = maxc;
  return want < 1 ? 1 : want;
}

int direct_sum(const double* x, int n, int n_el, const int64_t* targets,
               int nt, const WalkParams& wp, int nchunks, double4* partial,
               double* f, double* epot, cudaStream_t st) {
  if (nt == 0 || n == 0) return 0;
  int chunk = (n + nchunks - 1) / nchunks;
  chunk = (chunk + kDirT - 1) / kDirT * kDirT;
  int nch = (n + chunk - 1) / chunk;
  dim3 grid((nt + kDirT - 1) / kDirT, nch);
  if (wp.physics == 0)
    k_direct<0><<<grid, kDirT, 0, st>>>(x, n, n_el, targets, nt, chunk, wp, partial);
  else
    k_direct<1><<<grid, kDirT, 0, st>>>(x, n, n_el, targets, nt, chunk, wp, partial);
  k_direct_reduce<<<(nt + 255) / 256, 256, 0, st>>>(partial, nt, nch, f, epot);
  return 2;
}

}  // namespace tg
