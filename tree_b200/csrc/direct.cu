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

// ------------------------------------------------ allocation-free variant ----
// tree_gpu_direct_static: the same direct sum for callers that cannot
// allocate device memory.  Its scratch -- a validated copy of the target
// list, the per-chunk partial sums and an error word -- lives in one
// file-scope array that every GPU loading this library holds until exit.
#include <mutex>
#include "../../include/tree_gpu.h"

namespace {

constexpr size_t kStaticBytes = 8u << 20;         // 8 MiB per device
constexpr size_t kStaticFlagBytes = 256;          // error word (+ padding)
constexpr size_t kStaticTargetBytes = (size_t)TREE_GPU_DIRECT_STATIC_MAX_TARGETS * sizeof(int64_t);
constexpr size_t kStaticPartials =
    (kStaticBytes - kStaticFlagBytes - kStaticTargetBytes) / sizeof(double4);

__device__ __align__(256) unsigned char g_direct_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};

// Copies the targets into the scratch, replacing any index outside [0, n) by
// 0 and raising the error word, so the sum never reads out of bounds.
__global__ void k_sanitize_targets(const int64_t* __restrict__ in, int nt,
                                   int64_t n, int64_t* __restrict__ out,
                                   int32_t* flag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  int64_t v = in[t];
  if (v < 0 || v >= n) {
    atomicOr(flag, 1);
    v = 0;
  }
  out[t] = v;
}

// Address of the scratch on the current device, looked up once per device.
unsigned char* scratch_for_current_device(int* status) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *status = TREE_GPU_ERR_CUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_direct_scratch) != cudaSuccess || !p) {
      *status = TREE_GPU_ERR_CUDA;
      return nullptr;
    }
    g_scratch_ptr[dev] = (unsigned char*)p;
  }
  *status = TREE_GPU_OK;
  return g_scratch_ptr[dev];
}

double kelbg_lambda_um_static(double mu_amu, double te) {
  return 1.054571817e-34 / sqrt(2.0 * mu_amu * 1.66053906660e-27 * 1.380649e-23 * te) * 1e6;
}

// The launches of the allocation-free call, each returning its own status.
cudaError_t launch_sanitize(const int64_t* in, int nt, int64_t n, int64_t* out,
                            int32_t* flag, cudaStream_t st) {
  void* args[] = {(void*)&in, (void*)&nt, (void*)&n, (void*)&out, (void*)&flag};
  return cudaLaunchKernel((const void*)k_sanitize_targets, dim3((nt + 255) / 256),
                          dim3(256), args, 0, st);
}

cudaError_t launch_direct(const double* x, int n, int n_el, const int64_t* targets,
                          int nt, tg::WalkParams wp, int nchunks, double4* partial,
                          double* f, double* epot, cudaStream_t st) {
  // the grid of tg::direct_sum: tiles of kDirT targets x source chunks
  int chunk = (n + nchunks - 1) / nchunks;
  chunk = (chunk + tg::kDirT - 1) / tg::kDirT * tg::kDirT;
  const int nch = (n + chunk - 1) / chunk;
  const dim3 grid((nt + tg::kDirT - 1) / tg::kDirT, nch);
  void* a1[] = {(void*)&x, (void*)&n, (void*)&n_el, (void*)&targets, (void*)&nt,
                (void*)&chunk, (void*)&wp, (void*)&partial};
  const void* kfn = wp.physics == 0 ? (const void*)tg::k_direct<0> : (const void*)tg::k_direct<1>;
  cudaError_t e = cudaLaunchKernel(kfn, grid, dim3(tg::kDirT), a1, 0, st);
  if (e != cudaSuccess) return e;
  int nchv = nch;
  void* a2[] = {(void*)&partial, (void*)&nt, (void*)&nchv, (void*)&f, (void*)&epot};
  return cudaLaunchKernel((const void*)tg::k_direct_reduce, dim3((nt + 255) / 256),
                          dim3(256), a2, 0, st);
}

}  // namespace

extern "C" int tree_gpu_direct_static(const double* d_x, int64_t n_el,
                                      int64_t n_ion,
                                      const tree_gpu_params* params,
                                      const int64_t* d_targets, int64_t nt,
                                      double* d_f, double* d_epot,
                                      void* stream) {
  if (!params || n_el < 0 || n_ion < 0 || n_el + n_ion > 0x7fffffff || nt < 0)
    return TREE_GPU_ERR_ARG;
  if (nt > TREE_GPU_DIRECT_STATIC_MAX_TARGETS) return TREE_GPU_ERR_CAPACITY;
  if (params->physics != TREE_GPU_PHYS_REF && params->physics != TREE_GPU_PHYS_KELBG)
    return TREE_GPU_ERR_ARG;
  if (params->physics == TREE_GPU_PHYS_REF && !(params->rs > 0.0)) return TREE_GPU_ERR_ARG;
  if (params->physics == TREE_GPU_PHYS_KELBG &&
      !(params->te > 0.0 && params->xm_el > 0.0 && params->xm_ion > 0.0))
    return TREE_GPU_ERR_ARG;
  if (nt == 0) return TREE_GPU_OK;
  const int64_t n = n_el + n_ion;
  if (n == 0 || !d_x || !d_targets || !d_f || !d_epot) return TREE_GPU_ERR_ARG;
  int status = TREE_GPU_OK;
  unsigned char* base = scratch_for_current_device(&status);
  if (!base) return status;
  int32_t* flag = (int32_t*)base;
  int64_t* targets = (int64_t*)(base + kStaticFlagBytes);
  double4* partial = (double4*)(base + kStaticFlagBytes + kStaticTargetBytes);

  tg::WalkParams wp{};
  wp.physics = params->physics;
  wp.theta = params->theta;
  wp.rs = params->rs;
  if (params->physics == TREE_GPU_PHYS_KELBG) {
    const double me = params->xm_el, mi = params->xm_ion;
    wp.lam_ee = kelbg_lambda_um_static(me / 2.0, params->te);
    wp.lam_ei = kelbg_lambda_um_static(me * mi / (me + mi), params->te);
    wp.lam_ii = kelbg_lambda_um_static(mi / 2.0, params->te);
  }
  wp.dx_ei = params->dx_ei;
  wp.dx_ii = params->dx_ii;

  int nch = tg::direct_chunks((int)n, (int)nt);
  const int64_t fit = (int64_t)kStaticPartials / nt;
  if (nch > fit) nch = (int)fit;
  cudaStream_t st = (cudaStream_t)stream;
  // the error word keeps the previous call's value: clear it first
  if (cudaMemsetAsync(flag, 0, sizeof(int32_t), st) != cudaSuccess) return TREE_GPU_ERR_CUDA;
  // Each launch reports its own status (cudaLaunchKernel), so an error left
  // behind by the caller's earlier work is neither reported as this call's
  // nor cleared.
  if (launch_sanitize(d_targets, (int)nt, n, targets, flag, st) != cudaSuccess ||
      launch_direct(d_x, (int)n, (int)n_el, targets, (int)nt, wp, nch, partial, d_f,
                    d_epot, st) != cudaSuccess)
    return TREE_GPU_ERR_CUDA;
  int32_t hflag = 0;
  if (cudaMemcpyAsync(&hflag, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return TREE_GPU_ERR_CUDA;
  return hflag ? TREE_GPU_ERR_ARG : TREE_GPU_OK;
}
