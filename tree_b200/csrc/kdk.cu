// kdk.cu -- velocity Verlet on the device (compiled -fmad=false) and the
// deterministic reductions of the diagnostics.
//
// VVerletNotemp1 (vverlet.f90:24-39): v += 0.5*dt*f/m ; x += dt*v.
// VVerletNotemp2 (vverlet.f90:64-76): v += 0.5*dt*f/m, and on sample steps
// mv2 = sum m v^2, rad = sum m (x.v)^2/|x|^2 (vverlet.f90:81-106).
// Between two force evaluations the second half kick of step k and the first
// half kick + drift of step k+1 are one pass over memory (k_kick_kick_drift);
// the two half kicks stay two roundings, exactly as the reference does them.
#include "internal.cuh"
#include "kdk.h"

namespace tg {

constexpr int kKdkThreads = 256;

__device__ __forceinline__ void ke_terms(const double* xi, const double* vi,
                                         double xm, double& mv2, double& rad) {
  mv2 = xm * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
  double xv = xi[0] * vi[0] + xi[1] * vi[1] + xi[2] * vi[2];
  rad = xm * (xv * xv) / (xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
}

// Block sums of 4 values in fixed order (deterministic): partial[b*4 + j].
__device__ __forceinline__ void block_sum4(double a[4], double* partial) {
  __shared__ double sh[kKdkThreads / 32][4];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    for (int o = 16; o > 0; o >>= 1) a[j] += __shfl_down_sync(0xffffffffu, a[j], o);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < 4; ++j) sh[w][j] = a[j];
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0.0;
    for (int ww = 0; ww < kKdkThreads / 32; ++ww) s += sh[ww][threadIdx.x];
    partial[4 * blockIdx.x + threadIdx.x] = s;
  }
}

// Species of particle i: electrons [0, n_el) or, for an ensemble of clouds,
// the per-particle flag.
__device__ __forceinline__ bool is_ion(const uint8_t* __restrict__ ion, int i, int n_el) {
  return ion ? ion[i] != 0 : i >= n_el;
}

__global__ void k_kick_drift(double* __restrict__ x, double* __restrict__ v,
                             const double* __restrict__ f, int n, int n_el,
                             const uint8_t* __restrict__ ion, double dt,
                             double xm_e, double xm_i) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xm = is_ion(ion, i, n_el) ? xm_i : xm_e;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int64_t j = 3 * (int64_t)i + k;
    double vv = v[j] + 0.5 * dt * f[j] / xm;
    v[j] = vv;
    x[j] = x[j] + dt * vv;
  }
}

// Second half kick (+ kinetic sums of the kicked state when `sample`), then,
// when `drift`, the next step's first half kick and drift.
template <bool SAMPLE, bool DRIFT>
__global__ void __launch_bounds__(kKdkThreads)
    k_kick2(double* __restrict__ x, double* __restrict__ v,
            const double* __restrict__ f, int n, int n_el,
            const uint8_t* __restrict__ ion, double dt, double xm_e,
            double xm_i, double* __restrict__ partial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < n) {
    const bool is = is_ion(ion, i, n_el);
    double xm = is ? xm_i : xm_e;
    double xi[3], vi[3], fi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      int64_t j = 3 * (int64_t)i + k;
      xi[k] = x[j];
      vi[k] = v[j];
      fi[k] = f[j];
      vi[k] = vi[k] + 0.5 * dt * fi[k] / xm;  // VVerletNotemp2
    }
    if (SAMPLE) {
      double mv2, rad;
      ke_terms(xi, vi, xm, mv2, rad);
      int s = is ? 1 : 0;
      acc[2 * s] = mv2;
      acc[2 * s + 1] = rad;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      int64_t j = 3 * (int64_t)i + k;
      if (DRIFT) {
        vi[k] = vi[k] + 0.5 * dt * fi[k] / xm;  // next VVerletNotemp1
        x[j] = xi[k] + dt * vi[k];
      }
      v[j] = vi[k];
    }
  }
  if (SAMPLE) block_sum4(acc, partial);
}

// Sums rows of `partial` (nb x 4) in fixed order into out[0..3].  With cnt
// (the walk's interaction counters of this step in cnt[0..3] and cnt[8]),
// also adds them to the running totals cnt[4..7] and cnt[9].
__global__ void k_sum_partials4(const double* __restrict__ partial, int nb,
                                double* out, unsigned long long* cnt = nullptr) {
  __shared__ double sh[kKdkThreads];
  for (int j = 0; j < 4; ++j) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[4 * b + j];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
    __syncthreads();
  }
  if (cnt && threadIdx.x < 4) cnt[4 + threadIdx.x] += cnt[threadIdx.x];
  if (cnt && threadIdx.x == 4) cnt[9] += cnt[8];
}

// Potential energy: epot_part[i] = (contribution to Epot_e, to Epot_i).
__global__ void __launch_bounds__(kKdkThreads)
    k_epot_partial(const double2* __restrict__ ep, int n, double* partial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < n) {
    double2 e = ep[i];
    acc[0] = e.x;
    acc[1] = e.y;
  }
  block_sum4(acc, partial);
}

int kdk_partials_needed(int n) { return (n + kKdkThreads - 1) / kKdkThreads; }

void kick_drift(double* x, double* v, const double* f, int n, int n_el,
                const uint8_t* ion, double dt, double xm_e, double xm_i,
                cudaStream_t st) {
  if (n == 0) return;
  int g = (n + kKdkThreads - 1) / kKdkThreads;
  k_kick_drift<<<g, kKdkThreads, 0, st>>>(x, v, f, n, n_el, ion, dt, xm_e, xm_i);
}

void kick2(double* x, double* v, const double* f, int n, int n_el,
           const uint8_t* ion, double dt, double xm_e, double xm_i, bool sample,
           bool drift, double* partial, double* out4, cudaStream_t st) {
  if (n == 0) return;
  int g = (n + kKdkThreads - 1) / kKdkThreads;
  if (sample) {
    if (drift) k_kick2<true, true><<<g, kKdkThreads, 0, st>>>(x, v, f, n, n_el, ion, dt, xm_e, xm_i, partial);
    else k_kick2<true, false><<<g, kKdkThreads, 0, st>>>(x, v, f, n, n_el, ion, dt, xm_e, xm_i, partial);
    k_sum_partials4<<<1, kKdkThreads, 0, st>>>(partial, g, out4);
  } else {
    if (drift) k_kick2<false, true><<<g, kKdkThreads, 0, st>>>(x, v, f, n, n_el, ion, dt, xm_e, xm_i, partial);
    else k_kick2<false, false><<<g, kKdkThreads, 0, st>>>(x, v, f, n, n_el, ion, dt, xm_e, xm_i, partial);
  }
}

// Per-cloud diagnostics of an ensemble, one block per cloud in fixed order:
// out[6c..6c+5] = (Epot_e, Epot_i, mv2_el, mv2_ion, rad_el, rad_ion).
__global__ void __launch_bounds__(kKdkThreads)
    k_cloud_sums(const double* __restrict__ x, const double* __restrict__ v,
                 const double2* __restrict__ ep, const int32_t* __restrict__ start,
                 const int32_t* __restrict__ elec_end, double xm_e, double xm_i,
                 double* out) {
  __shared__ double sh[kKdkThreads / 32][6];
  const int c = blockIdx.x;
  const int i0 = start[c], i1 = start[c + 1], ie = elec_end[c];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const double2 e = ep[i];
    a[0] += e.x;
    a[1] += e.y;
    const int s = i >= ie;
    double mv2, rad;
    ke_terms(x + 3 * (int64_t)i, v + 3 * (int64_t)i, s ? xm_i : xm_e, mv2, rad);
    a[2 + s] += mv2;
    a[4 + s] += rad;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    for (int o = 16; o > 0; o >>= 1) a[j] += __shfl_down_sync(0xffffffffu, a[j], o);
    if (lane == 0) sh[w][j] = a[j];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int ww = 0; ww < kKdkThreads / 32; ++ww) s += sh[ww][threadIdx.x];
    out[6 * c + threadIdx.x] = s;
  }
}

void cloud_sums(const double* x, const double* v, const double2* ep,
                const int32_t* start, const int32_t* elec_end, int nseg,
                double xm_e, double xm_i, double* out, cudaStream_t st) {
  if (nseg > 0)
    k_cloud_sums<<<nseg, kKdkThreads, 0, st>>>(x, v, ep, start, elec_end, xm_e, xm_i, out);
}

void epot_sum(const double2* ep, int n, double* partial, double* out4,
              unsigned long long* counters, cudaStream_t st) {
  if (n == 0) {
    cudaMemsetAsync(out4, 0, 4 * sizeof(double), st);
    return;
  }
  int g = (n + kKdkThreads - 1) / kKdkThreads;
  k_epot_partial<<<g, kKdkThreads, 0, st>>>(ep, n, partial);
  k_sum_partials4<<<1, kKdkThreads, 0, st>>>(partial, g, out4, counters);
}

__global__ void k_sample_append(const double* __restrict__ diag, double* series,
                                int32_t* count, int cap) {
  if (threadIdx.x != 0) return;
  const int k = *count;
  if (k >= cap) return;
  double* r = series + 6 * (int64_t)k;
  r[0] = diag[0];  // Epot_e
  r[1] = diag[1];  // Epot_i
  r[2] = diag[4];  // mv2_el
  r[3] = diag[6];  // mv2_ion
  r[4] = diag[5];  // rad_el
  r[5] = diag[7];  // rad_ion
  *count = k + 1;
}

__global__ void k_rdf_fold(const uint32_t* __restrict__ bins32,
                           unsigned long long* acc64, int nbins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nbins) acc64[i] += bins32[i];
}

void sample_append(const double* diag, double* series, int32_t* count, int cap,
                   cudaStream_t st) {
  k_sample_append<<<1, 32, 0, st>>>(diag, series, count, cap);
}

void rdf_fold(const uint32_t* bins32, unsigned long long* acc64, cudaStream_t st) {
  const int nb = 2 * kRdfBins;
  k_rdf_fold<<<(nb + 255) / 256, 256, 0, st>>>(bins32, acc64, nb);
}

}  // namespace tg
