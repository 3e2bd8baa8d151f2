// build.cu -- device octree build for both species (compiled -fmad=false).
//
// The reference inserts particles one by one into a pointer octree
// (Insert_Tree_e/_i, tree.f90:103-447).  A particle's path depends only on
// comparisons against geometric centres that are themselves produced by
// repeated FP64 additions c_child = c + (+-0.25)*lx (tree.f90:123-126), so the
// reference tree is independent of insertion order and equals the trie of
// per-particle "replayed" paths cut at the first level where a particle is
// alone.  This file:
//   1. reduces the per-species bounding box (tree.f90:52-63),
//   2. replays each particle's path for 42 levels into a 128-bit key (3 bits
//      per level, child digit = bx + 2 by + 4 bz, the reference's bias-1),
//      with the species in bit 127,
//   3. sorts (key, index) with an LSD radix sort (8-bit digits),
//   4. derives the reference topology from adjacent common-prefix lengths and
//      emits nodes directly in pre-order (children 1..8 = the reference's
//      recursion order) with subtree-skip links,
//   5. computes the one-level moments of PSeudoE/PSeudoI (tree.f90:450-659)
//      bottom-up with per-node arrival counters, in the reference's child
//      order and operation order, so FP64 values are bit-identical.
#include <cstdio>
#include "internal.cuh"
#include "build.h"

namespace tg {

// ---------------------------------------------------------------- bbox ----
__global__ void k_bbox_init(uint64_t* bb, int32_t* err) {
  int t = threadIdx.x;
  if (t < 12) bb[t] = (t & 1) ? 0ull : ~0ull;
  if (t == 0) *err = 0;
}

__device__ __forceinline__ uint64_t shfl_min_u64(uint64_t v) {
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}
__device__ __forceinline__ uint64_t shfl_max_u64(uint64_t v) {
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// bb[(s*3+k)*2 + 0] = ord(min), +1 = ord(max)
__global__ void k_bbox(const double* __restrict__ x, int n, int n_el,
                       uint64_t* bb, int32_t* err) {
  uint64_t mn[2][3], mx[2][3];
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      mn[s][k] = ~0ull;
      mx[s][k] = 0ull;
    }
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    int s = i >= n_el;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * (int64_t)i + k];
      if (!isfinite(v)) bad = true;
      uint64_t o = ord_from_double(v);
      if (s == 0) {
        mn[0][k] = o < mn[0][k] ? o : mn[0][k];
        mx[0][k] = o > mx[0][k] ? o : mx[0][k];
      } else {
        mn[1][k] = o < mn[1][k] ? o : mn[1][k];
        mx[1][k] = o > mx[1][k] ? o : mx[1][k];
      }
    }
  }
  if (bad) set_error(err, kErrNonFinite);
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uint64_t a = shfl_min_u64(mn[s][k]);
      uint64_t b = shfl_max_u64(mx[s][k]);
      if ((threadIdx.x & 31) == 0) {
        if (a != ~0ull) atomicMin((unsigned long long*)&bb[(s * 3 + k) * 2], a);
        if (b != 0ull) atomicMax((unsigned long long*)&bb[(s * 3 + k) * 2 + 1], b);
      }
    }
}

// Root box per species: tree.f90:58-63 (xx = (max+min)/2, lx = max-min).
__global__ void k_geom(const uint64_t* bb, int n, int n_el, Geom* g) {
  int s = threadIdx.x;
  if (s >= 2) return;
  Geom G;
  G.n = s == 0 ? n_el : n - n_el;
  G.first = s == 0 ? 0 : n_el;
  double smax = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (G.n > 0) {
      double lo = double_from_ord(bb[(s * 3 + k) * 2]);
      double hi = double_from_ord(bb[(s * 3 + k) * 2 + 1]);
      G.c0[k] = (hi + lo) / 2.0;
      G.lx0[k] = hi - lo;
    } else {
      G.c0[k] = 0.0;
      G.lx0[k] = 0.0;
    }
    if (k == 0 || G.lx0[k] > smax) smax = G.lx0[k];
  }
  G.smax0 = smax;
  g[s] = G;
}

// Per-cloud bounding boxes: one block per cloud, bb[(c*3+k)*2 + 0/1] = ord
// of the min / max along axis k.
__global__ void k_bbox_seg(const double* __restrict__ x,
                           const int32_t* __restrict__ start, uint64_t* bb,
                           int32_t* err) {
  __shared__ uint64_t smin[3][256 / 32], smax[3][256 / 32];
  const int c = blockIdx.x;
  const int i0 = start[c], i1 = start[c + 1];
  uint64_t mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0ull, 0ull, 0ull};
  bool bad = false;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double v = x[3 * (int64_t)i + k];
      if (!isfinite(v)) bad = true;
      const uint64_t o = ord_from_double(v);
      mn[k] = o < mn[k] ? o : mn[k];
      mx[k] = o > mx[k] ? o : mx[k];
    }
  if (bad) set_error(err, kErrNonFinite);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint64_t a = shfl_min_u64(mn[k]), b = shfl_max_u64(mx[k]);
    if (lane == 0) {
      smin[k][w] = a;
      smax[k][w] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int k = threadIdx.x;
    uint64_t a = ~0ull, b = 0ull;
    for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) {
      a = smin[k][ww] < a ? smin[k][ww] : a;
      b = smax[k][ww] > b ? smax[k][ww] : b;
    }
    bb[(c * 3 + k) * 2] = a;
    bb[(c * 3 + k) * 2 + 1] = b;
  }
}

// Root box per cloud, as k_geom does per species.
__global__ void k_geom_seg(const uint64_t* bb, const int32_t* __restrict__ start,
                           int nseg, Geom* g) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nseg) return;
  Geom G;
  G.first = start[c];
  G.n = start[c + 1] - start[c];
  double smax = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (G.n > 0) {
      const double lo = double_from_ord(bb[(c * 3 + k) * 2]);
      const double hi = double_from_ord(bb[(c * 3 + k) * 2 + 1]);
      G.c0[k] = (hi + lo) / 2.0;
      G.lx0[k] = hi - lo;
    } else {
      G.c0[k] = 0.0;
      G.lx0[k] = 0.0;
    }
    if (k == 0 || G.lx0[k] > smax) smax = G.lx0[k];
  }
  G.smax0 = smax;
  g[c] = G;
}

// ---------------------------------------------------------------- keys ----
// Replays Insert_Tree's descent (tree.f90:132-173 comparisons, 123-126 child
// centres) for 42 levels.  The reference recursion has no depth limit; 42
// levels resolve 2^-42 of the root box, so clouds whose box has grown by
// orders of magnitude (escaping electrons) still separate every particle.
// Key layouts (level l = 1..42, digit d_l):
//   per-species trees (lsb = 0): bit 127 = species, d_l in bits
//     (127 - 3l) .. (125 - 3l), bit 0 = 0;
//   combined tree (lsb = 1): d_l in bits (128 - 3l) .. (126 - 3l), bit 1 = 0,
//     bit 0 = species, a 43rd one-bit level that separates an electron
//     sitting exactly on an ion (the t = 0 state of the clouds).
// In both, the digit of level l is (key >> (127 - 3l + lsb)) & 7.
// An ensemble of clouds (combined layout) puts the cloud id in the top `top`
// bits and keeps nlev = (126 - top) / 3 spatial levels right below it (any
// spare bits sit between level nlev and the species bit); the digit of level
// l is then (key >> (128 - top - 3l)) & 7, which is the general form
// (top = 1 - lsb for the single-cloud layouts).
__global__ void k_keys(const double* __restrict__ x, int n, int n_el,
                       int lsb, int n_el_charge, const Geom* __restrict__ geom,
                       Ensemble ens, key128* keys, uint64_t* hi, uint32_t* vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = i >= n_el;
  int seg = s, top = 1 - lsb, nlev = kMaxLevel;
  bool ion = i >= n_el_charge;
  if (ens.nseg > 0) {
    seg = seg_of(ens.start, ens.nseg, i);
    ion = i >= __ldg(&ens.elec_end[seg]);
    top = ens.top;
    nlev = ens.nlev;
  }
  const Geom& G = geom[seg];
  double p[3], c[3], lx[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[k] = x[3 * (int64_t)i + k];
    c[k] = G.c0[k];
    lx[k] = G.lx0[k];
  }
  key128 key = 0;
  for (int l = 0; l < nlev; ++l) {
    uint32_t b = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      bool hi = !(p[k] < c[k]);
      b |= (uint32_t)hi << k;
      c[k] = c[k] + (hi ? 0.25 : -0.25) * lx[k];
      lx[k] = lx[k] * 0.5;
    }
    key = (key << 3) | (key128)b;
  }
  // level 1 right below the top bits; the bits under level nlev are zero
  // except, in the combined layout, the species in bit 0
  key <<= (128 - top - 3 * nlev);
  if (lsb) key |= (key128)(ion ? 1u : 0u);
  if (top > 0) key |= (key128)(uint32_t)seg << (128 - top);
  keys[i] = key;
  hi[i] = (uint64_t)(key >> 64);
  vals[i] = (uint32_t)i;
}

// Full keys in the order of the sorted high words.
__global__ void k_gather_keys(const key128* __restrict__ keys_in,
                              const uint32_t* __restrict__ vals, int n, key128* keys_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) keys_out[p] = keys_in[vals[p]];
}

// ---------------------------------------------------------------- scan ----
// Exclusive scan of int32 with block partials (three phases, no inter-block
// waiting).  out[n] receives the total when `write_total`.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t* total) {
  __shared__ int32_t warp_sums[kScanThreads / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (w == 0) {
    int32_t ws = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
    int32_t wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - ws;
    if (lane == kScanThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  int32_t r = inc - v + warp_sums[w];
  __syncthreads();
  return r;
}

__global__ void k_scan_reduce(const int32_t* __restrict__ in, int n,
                              int32_t* partial) {
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  int32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  __shared__ int32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_scan_partials(int32_t* partial, int nb) {
  __shared__ int32_t carry_s;
  __shared__ int32_t tot;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanThreads) {
    int i = base + threadIdx.x;
    int32_t v = i < nb ? partial[i] : 0;
    int32_t e = block_excl_scan(v, &tot);
    int32_t carry = carry_s;
    if (i < nb) partial[i] = e + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nb] = carry_s;
}

__global__ void k_scan_down(const int32_t* __restrict__ in, int n,
                            const int32_t* __restrict__ partial, int32_t* out,
                            int write_total) {
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  // each thread owns kScanItems consecutive elements
  int32_t v[kScanItems];
  int32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + j;
    v[j] = i < n ? in[i] : 0;
    s += v[j];
  }
  __shared__ int32_t tot;
  int32_t e = block_excl_scan(s, &tot) + partial[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + j;
    if (i < n) out[i] = e;
    e += v[j];
  }
  if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    out[n] = partial[gridDim.x];
}

// note: k_scan_reduce sums strided elements while k_scan_down scans
// contiguous runs; both cover exactly the tile [base, base+kScanTile).

int scan_partials_needed(int n) { return (n + kScanTile - 1) / kScanTile + 1; }

int exclusive_scan(const int32_t* in, int32_t* out, int n, int32_t* partial,
                   bool write_total, cudaStream_t st) {
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    if (write_total) cudaMemsetAsync(out, 0, sizeof(int32_t), st);
    return 0;
  }
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, n, partial);
  k_scan_partials<<<1, kScanThreads, 0, st>>>(partial, nb);
  k_scan_down<<<nb, kScanThreads, 0, st>>>(in, n, partial, out,
                                           write_total ? 1 : 0);
  return 3;
}

// ---------------------------------------------------------- radix sort ----
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsIters = 8;                        // items per lane
constexpr int kRsTile = kRsThreads * kRsIters;     // 2048 items per block
constexpr int kRsBins = 256;

int radix_blocks(int n) { return (n + kRsTile - 1) / kRsTile; }

template <class K>
__global__ void k_rs_hist(const K* __restrict__ keys, int n, int shift,
                          int32_t* hist /* [256][nb] */) {
  __shared__ int32_t h[kRsBins];
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int j = 0; j < kRsIters; ++j) {
    int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(int)((keys[i] >> shift) & 0xff)], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x)
    hist[(int64_t)b * gridDim.x + blockIdx.x] = h[b];
}

// Stable scatter: tile order is warp-major (warp w owns items
// [w*32*kRsIters, (w+1)*32*kRsIters) of the tile), then iteration, then lane.
template <class K>
__global__ void __launch_bounds__(kRsThreads)
    k_rs_scatter(const K* __restrict__ keys_in,
                 const uint32_t* __restrict__ vals_in, int n, int shift,
                 const int32_t* __restrict__ offs /* scanned [256][nb] */,
                 K* __restrict__ keys_out,
                 uint32_t* __restrict__ vals_out) {
  __shared__ int32_t whist[kRsWarps][kRsBins];
  __shared__ int32_t base_s[kRsBins];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) {
    base_s[b] = offs[(int64_t)b * gridDim.x + blockIdx.x];
#pragma unroll
    for (int ww = 0; ww < kRsWarps; ++ww) whist[ww][b] = 0;
  }
  __syncthreads();
  int64_t wbase = (int64_t)blockIdx.x * kRsTile + (int64_t)w * (32 * kRsIters);
  K k[kRsIters];
  uint32_t v[kRsIters];
  int32_t loc[kRsIters];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kRsIters; ++j) {
    int64_t i = wbase + j * 32 + lane;
    bool ok = i < n;
    k[j] = ok ? keys_in[i] : (K)0;
    v[j] = ok ? vals_in[i] : 0u;
    int d = ok ? (int)((k[j] >> shift) & 0xff) : kRsBins;  // sentinel bin
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & lt);
    int32_t before = ok ? whist[w][d] : 0;
    __syncwarp();
    if (ok && rank == 0) whist[w][d] = before + __popc(peers);
    __syncwarp();
    loc[j] = ok ? before + rank : -1;
  }
  __syncthreads();
  // exclusive prefix over warps per digit
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) {
    int32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kRsWarps; ++ww) {
      int32_t t = whist[ww][b];
      whist[ww][b] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kRsIters; ++j) {
    if (loc[j] < 0) continue;
    int d = (int)((k[j] >> shift) & 0xff);
    int64_t pos = (int64_t)base_s[d] + whist[w][d] + loc[j];
    keys_out[pos] = k[j];
    vals_out[pos] = v[j];
  }
}

// Sorts (keys, vals) in place using the alternate buffers; an even number of
// 8-bit passes, so the result ends in the primary buffers.
template <class K>
int radix_sort(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int n,
               int32_t* hist, int32_t* partial, cudaStream_t st, int first_byte) {
  if (n <= 1) return 0;
  int launches = 0;
  int nb = radix_blocks(n);
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int pass = first_byte; pass < (int)sizeof(K); ++pass) {
    int shift = pass * 8;
    k_rs_hist<K><<<nb, kRsThreads, 0, st>>>(kin, n, shift, hist);
    launches += 2 + exclusive_scan(hist, hist, kRsBins * nb, partial, false, st);
    k_rs_scatter<K><<<nb, kRsThreads, 0, st>>>(kin, vin, n, shift, hist, kout,
                                               vout);
    K* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
  }
  return launches;
}

template int radix_sort<uint64_t>(uint64_t*, uint32_t*, uint64_t*, uint32_t*, int,
                                  int32_t*, int32_t*, cudaStream_t, int);
template int radix_sort<key128>(key128*, uint32_t*, key128*, uint32_t*, int,
                                int32_t*, int32_t*, cudaStream_t, int);

// After a stable sort on the high 64 key bits, runs of equal high words
// (particles closer than about 2^-21 of the root box: co-located e-i pairs,
// tight pairs) are put in full-key order by one thread per run.  Runs are
// short (typically 2), and equal full keys keep their stable order.  A run
// longer than kTieSerial (a tight cluster in a box stretched by a far
// outlier) is left alone and raises *long_run, which makes k_sort_block sort
// the whole array by the full key; that sort is stable, so the result is the
// same order either way.
constexpr int kTieSerial = 64;

__global__ void k_tie_fix(key128* keys, uint32_t* vals, int n, int32_t* long_run) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p + 1 >= n) return;
  const uint64_t h = (uint64_t)(keys[p] >> 64);
  if ((uint64_t)(keys[p + 1] >> 64) != h) return;
  if (p > 0 && (uint64_t)(keys[p - 1] >> 64) == h) return;  // not the run start
  int e = p + 1;
  while (e < n && e - p <= kTieSerial && (uint64_t)(keys[e] >> 64) == h) ++e;
  if (e - p > kTieSerial) {
    *long_run = 1;
    return;
  }
  for (int i = p + 1; i < e; ++i) {  // insertion sort on the low word
    const key128 k = keys[i];
    const uint32_t v = vals[i];
    int j = i - 1;
    while (j >= p && keys[j] > k) {
      keys[j + 1] = keys[j];
      vals[j + 1] = vals[j];
      --j;
    }
    keys[j + 1] = k;
    vals[j + 1] = v;
  }
}

// Stable LSD radix sort of all 16 key bytes by ONE block of kSbThreads, run
// only when *gate != 0 (otherwise the launch returns at once): the rare
// fallback of the high-word sort, slow (one SM streams the array 32 times)
// but a single launch in the common case.  Same order rule as k_rs_scatter:
// per tile, warp w owns items [w*kSbItems*32, (w+1)*kSbItems*32).
constexpr int kSbThreads = 1024;
constexpr int kSbWarps = kSbThreads / 32;
constexpr int kSbItems = 4;
constexpr int kSbTile = kSbThreads * kSbItems;

__global__ void __launch_bounds__(kSbThreads)
    k_sort_block(key128* keys, uint32_t* vals, key128* keys_alt, uint32_t* vals_alt,
                 int n, const int32_t* gate) {
  if (*gate == 0) return;
  __shared__ int32_t whist[kSbWarps][kRsBins];
  __shared__ int32_t base_s[kRsBins];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  key128* kin = keys;
  uint32_t* vin = vals;
  key128* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int pass = 0; pass < 16; ++pass) {
    const int shift = 8 * pass;
    for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) base_s[b] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      atomicAdd(&base_s[(int)((kin[i] >> shift) & 0xff)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0;
      for (int b = 0; b < kRsBins; ++b) {
        const int t = base_s[b];
        base_s[b] = run;
        run += t;
      }
    }
    __syncthreads();
    for (int64_t tile = 0; tile < n; tile += kSbTile) {
      for (int b = threadIdx.x; b < kRsBins; b += blockDim.x)
#pragma unroll
        for (int ww = 0; ww < kSbWarps; ++ww) whist[ww][b] = 0;
      __syncthreads();
      const int64_t wbase = tile + (int64_t)w * (32 * kSbItems);
      key128 k[kSbItems];
      uint32_t v[kSbItems];
      int32_t loc[kSbItems];
#pragma unroll
      for (int j = 0; j < kSbItems; ++j) {
        const int64_t i = wbase + j * 32 + lane;
        const bool ok = i < n;
        k[j] = ok ? kin[i] : (key128)0;
        v[j] = ok ? vin[i] : 0u;
        const int d = ok ? (int)((k[j] >> shift) & 0xff) : kRsBins;  // sentinel bin
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        const int32_t before = ok ? whist[w][d] : 0;
        __syncwarp();
        if (ok && rank == 0) whist[w][d] = before + __popc(peers);
        __syncwarp();
        loc[j] = ok ? before + rank : -1;
      }
      __syncthreads();
      // exclusive prefix over warps per digit; the tile's totals advance base_s
      for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) {
        int32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < kSbWarps; ++ww) {
          const int32_t t = whist[ww][b];
          whist[ww][b] = run + base_s[b];
          run += t;
        }
        base_s[b] += run;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kSbItems; ++j) {
        if (loc[j] < 0) continue;
        const int d = (int)((k[j] >> shift) & 0xff);
        const int64_t pos = (int64_t)whist[w][d] + loc[j];
        kout[pos] = k[j];
        vout[pos] = v[j];
      }
      __syncthreads();
    }
    key128* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
  }
}

// ------------------------------------------------------------ topology ----
__device__ __forceinline__ int clz128(key128 x) {
  const uint64_t hi = (uint64_t)(x >> 64), lo = (uint64_t)x;
  return hi ? __clzll((long long)hi) : 64 + __clzll((long long)lo);
}

// L[p] = number of leading levels that sorted keys p and p+1 share (same
// species tree / same cloud: equal `top` bits), else -1.  Identical keys mean
// the level cap was hit.
__global__ void k_common_levels(const key128* __restrict__ keys, int n,
                                int top, int nlev, int8_t* L, int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int8_t r = -1;
  if (p + 1 < n) {
    key128 a = keys[p], b = keys[p + 1];
    key128 x = a ^ b;
    if (top == 0 || (x >> (128 - top)) == 0) {
      if (x == 0) {
        set_error(err, kErrDepth);
        r = (int8_t)nlev;
      } else {
        // lz >= top (same tree); for the combined layouts lz = 127 means only
        // the species bit differs, i.e. all nlev spatial levels are shared
        int lev = (clz128(x) - top) / 3;
        r = (int8_t)(lev < nlev ? lev : nlev);
      }
    }
  }
  L[p] = r;
}

__global__ void k_counts(const int8_t* __restrict__ L, int n, int32_t* cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  cnt[p] = (hi > lo ? hi - lo : 0) + 1;
}

// first q in [lo_i, hi_i) with (keys[q] >> sh) > pre ; keys sorted
__device__ __forceinline__ int upper_prefix(const key128* __restrict__ keys,
                                            int lo_i, int hi_i, int sh,
                                            key128 pre) {
  while (lo_i < hi_i) {
    int mid = lo_i + ((hi_i - lo_i) >> 1);
    if ((keys[mid] >> sh) > pre) hi_i = mid;
    else lo_i = mid + 1;
  }
  return lo_i;
}
// first q in [lo_i, hi_i) with (keys[q] >> sh) >= pre
__device__ __forceinline__ int lower_prefix(const key128* __restrict__ keys,
                                            int lo_i, int hi_i, int sh,
                                            key128 pre) {
  while (lo_i < hi_i) {
    int mid = lo_i + ((hi_i - lo_i) >> 1);
    if ((keys[mid] >> sh) >= pre) hi_i = mid;
    else lo_i = mid + 1;
  }
  return lo_i;
}

// Shift that leaves the first d levels of a key (with the top bits; 1 <= d <=
// nlev); level nlev + 1 of the combined layout is the whole key.
__device__ __forceinline__ int shift_for_level(int d, int top) {
  int s = 128 - top - 3 * d;
  return s > 0 ? s : 0;
}

// Ends of the level-d cell of particle p inside its segment [sb, se): keys q
// and q+1 share fewer than d levels exactly where the level-d prefix
// changes, so a short scan of the common-level array L finds the end of a
// small cell (most of them); the keys beyond the scanned window are
// binary-searched.  Both give the same index.
constexpr int kRangeScan = 32;

// first q in (p, se) outside the cell, or se
__device__ __forceinline__ int range_end(const key128* __restrict__ keys,
                                         const int8_t* __restrict__ L, int p, int se,
                                         int d, int sh, key128 pre) {
  const int lim = p + kRangeScan < se ? p + kRangeScan : se;
  for (int q = p + 1; q < lim; ++q)
    if (L[q - 1] < d) return q;
  return upper_prefix(keys, lim, se, sh, pre);
}

// first q in [sb, p] inside the cell (level 0: the segment's root cell)
__device__ __forceinline__ int range_start(const key128* __restrict__ keys,
                                           const int8_t* __restrict__ L, int sb, int p,
                                           int d, int sh, key128 pre) {
  if (d == 0) return sb;
  const int lim = p - kRangeScan > sb ? p - kRangeScan : sb;
  for (int j = p - 1; j >= lim; --j)
    if (L[j] < d) return j + 1;
  return lower_prefix(keys, sb, lim + 1, sh, pre);
}

// Index of the twig at level d that contains sorted particle p, given that it
// was opened at an earlier particle (first particle of the level-d prefix).
__device__ __forceinline__ int twig_index_before(
    const key128* __restrict__ keys, const int8_t* __restrict__ L,
    const int32_t* __restrict__ off, int sb, int p, int d, int top) {
  const int sh = d > 0 ? shift_for_level(d, top) : 0;
  const key128 pre = d > 0 ? keys[p] >> sh : (key128)0;
  int q = range_start(keys, L, sb, p, d, sh, pre);
  int lo_q = q == 0 ? -1 : (int)L[q - 1];
  return off[q] + (d - lo_q - 1);
}

// Writes every node in pre-order.  node_c.xyz of twigs receives the
// geometric centre (replayed like k_keys); the upward pass replaces it.
__global__ void k_topology(const key128* __restrict__ keys,
                           const uint32_t* __restrict__ vals,
                           const int8_t* __restrict__ L,
                           const int32_t* __restrict__ off, int n, int n_el,
                           int lsb, const Geom* __restrict__ geom, int cap,
                           double4* node_c, int32_t* node_skip,
                           int32_t* node_pt, int32_t* node_parent,
                           int32_t* node_nchild, int32_t* node_done,
                           int8_t* node_level, MixedNodes mx, Ensemble ens,
                           int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  int s = p >= n_el;
  int sb = s ? n_el : 0, se = s ? n : n_el;
  int top = 1 - lsb, nlev = kMaxLevel;
  if (ens.nseg > 0) {  // sorted order keeps every cloud's index range
    s = seg_of(ens.start, ens.nseg, p);
    sb = ens.start[s];
    se = ens.start[s + 1];
    top = ens.top;
    nlev = ens.nlev;
  }
  int tree_end = off[se];
  int base = off[p];
  key128 key = keys[p];
  const Geom& G = geom[s];
  double c[3], lx[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c[k] = G.c0[k];
    lx[k] = G.lx0[k];
  }
  for (int d = 0; d <= hi; ++d) {
    if (d >= lo + 1) {
      int idx = base + (d - lo - 1);
      if (idx >= cap) {
        set_error(err, kErrCapacity);
        return;
      }
      node_c[idx] = make_double4(c[0], c[1], c[2], 0.0);
      node_level[idx] = (int8_t)d;
      node_pt[idx] = -1;
      node_done[idx] = 0;
      node_nchild[idx] = 0;  // children add themselves below (other threads
                             // add after this store: see k_link_children)
      int sk, q_end;
      if (d == 0) {
        sk = tree_end;
        q_end = se;
      } else {
        int sh = shift_for_level(d, top);
        int q = range_end(keys, L, p, se, d, sh, key >> sh);
        sk = q < se ? off[q] : tree_end;
        q_end = q;
      }
      node_skip[idx] = sk;
      // particle range and child table used by the mixed-precision walk
      mx.first[idx] = p;
      mx.count[idx] = q_end - p;
      mx.digit[idx] = d == 0 ? (int8_t)0 : (int8_t)((key >> (128 - top - 3 * d)) & 7);
      int4* kk = reinterpret_cast<int4*>(mx.kids + 8 * (int64_t)idx);
      kk[0] = make_int4(-1, -1, -1, -1);
      kk[1] = make_int4(-1, -1, -1, -1);
      int par;
      if (d == 0) par = -1;
      else if (d > lo + 1) par = idx - 1;
      else par = twig_index_before(keys, L, off, sb, p, d - 1, top);
      node_parent[idx] = par;
    }
    // descend one level along this particle's digits
    if (d < nlev) {
      int dig = (int)((key >> (125 - top - 3 * d)) & 7);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        bool bit = (dig >> k) & 1;
        c[k] = c[k] + (bit ? 0.25 : -0.25) * lx[k];
        lx[k] = lx[k] * 0.5;
      }
    }
  }
  int ntw = hi > lo ? hi - lo : 0;
  int leaf = base + ntw;
  if (leaf >= cap) {
    set_error(err, kErrCapacity);
    return;
  }
  int depth = (lo > hi ? lo : hi) + 1;
  node_level[leaf] = (int8_t)depth;
  node_skip[leaf] = leaf + 1;
  node_pt[leaf] = (int32_t)vals[p];
  node_done[leaf] = 0;
  node_nchild[leaf] = 0;
  mx.first[leaf] = p;
  mx.count[leaf] = 1;
  mx.digit[leaf] = depth <= nlev ? (int8_t)((key >> (128 - top - 3 * depth)) & 7)
                                 : (int8_t)(lsb ? (int)(key & 1) : 0);
  node_parent[leaf] = ntw > 0 ? leaf - 1
                              : twig_index_before(keys, L, off, sb, p, depth - 1, top);
}

// ------------------------------------------- combined-tree topology ----
// The combined tree of the mixed path is written one thread per node rather
// than one per particle: no lane waits on another's emission loop.  Node i
// belongs to the sorted particle that emits it (owner[i]); its slot among
// that particle's nodes gives its level.  Twig centres are the closed form
// of the key's digits, c_k = c0_k + lx0_k ((B_k + 1/2) 2^-d - 1/2), B_k the
// d bits of axis k (within a rounding of the level-by-level descent; the
// mixed walk reads them only through |centroid - centre|).  Leaves also
// write their position (w = -1, the walk's leaf mark) and the sorted copy
// xs (w = 1 for ions).  The child table is cleared here and filled by
// k_link_children; per-node skip and child counts are not needed.
__global__ void k_owner(const int32_t* __restrict__ off, int n, int cap, int32_t* owner) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int e = off[p + 1] < cap ? off[p + 1] : cap;
  for (int i = off[p]; i < e; ++i) owner[i] = p;
}

__device__ __forceinline__ void topology_node(
    int i, const key128* __restrict__ keys, const uint32_t* __restrict__ vals,
    const int8_t* __restrict__ L, const int32_t* __restrict__ off,
    const int32_t* __restrict__ owner, int n, int n_el_charge, const double* __restrict__ x,
    const Geom* __restrict__ geom, double4* node_c, int32_t* node_pt, int32_t* node_parent,
    int32_t* node_done, int8_t* node_level, const MixedNodes& mx, const Ensemble& ens) {
  const int p = owner[i];
  const int slot = i - off[p];
  int lo, hi;
  lo_hi(L, p, lo, hi);
  const int ntw = hi > lo ? hi - lo : 0;
  int s = 0, sb = 0, se = n, top = 0, nlev = kMaxLevel;  // single cloud: top = 1 - lsb = 0
  if (ens.nseg > 0) {
    s = seg_of(ens.start, ens.nseg, p);
    sb = ens.start[s];
    se = ens.start[s + 1];
    top = ens.top;
    nlev = ens.nlev;
  }
  const key128 key = keys[p];
  node_done[i] = 0;
  mx.first[i] = p;
  if (slot < ntw) {
    const int d = lo + 1 + slot;
    // axis bits of the first d digits (digit l at bits 127 - 3l .. 125 - 3l of key << top)
    uint64_t B[3] = {0, 0, 0};
    key128 kk = key << top;
    for (int l = 0; l < d; ++l) {
      const uint32_t dig = (uint32_t)(kk >> 125) & 7u;
      B[0] = 2 * B[0] + (dig & 1u);
      B[1] = 2 * B[1] + ((dig >> 1) & 1u);
      B[2] = 2 * B[2] + (dig >> 2);
      kk <<= 3;
    }
    const Geom& G = geom[s];
    double c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double f = ldexp((double)B[k] + 0.5, -d) - 0.5;  // exact
      c[k] = G.c0[k] + G.lx0[k] * f;
    }
    node_c[i] = make_double4(c[0], c[1], c[2], 0.0);
    node_level[i] = (int8_t)d;
    node_pt[i] = -1;
    int q_end = se;
    if (d > 0) {
      const int sh = shift_for_level(d, top);
      q_end = range_end(keys, L, p, se, d, sh, key >> sh);
    }
    mx.count[i] = q_end - p;
    mx.digit[i] = d == 0 ? (int8_t)0 : (int8_t)((key >> (128 - top - 3 * d)) & 7);
    int4* kk4 = reinterpret_cast<int4*>(mx.kids + 8 * (int64_t)i);
    kk4[0] = make_int4(-1, -1, -1, -1);
    kk4[1] = make_int4(-1, -1, -1, -1);
    node_parent[i] = d == 0 ? -1
                     : slot > 0 ? i - 1
                                : twig_index_before(keys, L, off, sb, p, d - 1, top);
  } else {
    const int depth = (lo > hi ? lo : hi) + 1;
    const uint32_t o = vals[p];
    node_level[i] = (int8_t)depth;
    node_pt[i] = (int32_t)o;
    mx.count[i] = 1;
    mx.digit[i] = depth <= nlev ? (int8_t)((key >> (128 - top - 3 * depth)) & 7)
                                : (int8_t)(key & 1);
    node_parent[i] = ntw > 0 ? i - 1 : twig_index_before(keys, L, off, sb, p, depth - 1, top);
    const bool ion = (int)o >= (ens.nseg > 0 ? __ldg(&ens.elec_end[s]) : n_el_charge);
    const double px = x[3 * (int64_t)o], py = x[3 * (int64_t)o + 1], pz = x[3 * (int64_t)o + 2];
    node_c[i] = make_double4(px, py, pz, -1.0);
    mx.xs[p] = make_double4(px, py, pz, ion ? 1.0 : 0.0);
  }
}

__global__ void k_topology_mixed(const key128* __restrict__ keys,
                                 const uint32_t* __restrict__ vals,
                                 const int8_t* __restrict__ L,
                                 const int32_t* __restrict__ off,
                                 const int32_t* __restrict__ owner,
                                 const int32_t* __restrict__ bounds, int n,
                                 int n_el_charge, const double* __restrict__ x,
                                 const Geom* __restrict__ geom, int cap, double4* node_c,
                                 int32_t* node_pt, int32_t* node_parent, int32_t* node_done,
                                 int8_t* node_level, MixedNodes mx, Ensemble ens) {
  const int m = bounds[2] < cap ? bounds[2] : cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    topology_node(i, keys, vals, L, off, owner, n, n_el_charge, x, geom, node_c, node_pt,
                  node_parent, node_done, node_level, mx, ens);
}

// Counts children per twig (separate launch so the zeroing in k_topology is
// complete).
__global__ void k_link_children(const int32_t* __restrict__ node_parent,
                                const int32_t* __restrict__ bounds, int cap,
                                int32_t* node_nchild, MixedNodes mx) {
  const int m = bounds[2] < cap ? bounds[2] : cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int par = node_parent[i];
    if (par >= 0) {
      if (node_nchild) atomicAdd(&node_nchild[par], 1);
      mx.kids[8 * (int64_t)par + mx.digit[i]] = i;  // siblings have distinct digits
    }
  }
}

// Root node of every cloud: the first node its first sorted particle emits.
__global__ void k_roots(const int32_t* __restrict__ off,
                        const int32_t* __restrict__ start, int nseg,
                        int32_t* roots) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nseg) roots[c] = off[start[c]];
}

__global__ void k_bounds(const int32_t* __restrict__ off, int n, int n_el,
                         int cap, int32_t* bounds, int32_t* err) {
  if (threadIdx.x != 0) return;
  int me = off[n_el], m = off[n];
  if (m > cap) {
    set_error(err, kErrCapacity);
    me = me < cap ? me : cap;
    m = cap;
  }
  bounds[0] = 0;
  bounds[1] = me;
  bounds[2] = m;
  bounds[3] = off[n];  // untruncated node count (for capacity growth)
}

// ------------------------------------------------------------- upward ----
// One thread per sorted particle: writes its leaf, then climbs while it is the
// last child to arrive, computing PSeudo's moments for each completed twig.
__global__ void k_upward(const double* __restrict__ x,
                         const uint32_t* __restrict__ vals,
                         const int8_t* __restrict__ L,
                         const int32_t* __restrict__ off, int n, int n_el,
                         const Geom* __restrict__ geom, double theta, int cap, const int32_t* __restrict__ bounds,
                         double4* node_c, double2* node_m,
                         const int32_t* __restrict__ node_skip,
                         const int32_t* __restrict__ node_parent,
                         const int32_t* __restrict__ node_nchild,
                         int32_t* node_done,
                         const int8_t* __restrict__ node_level, int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (*((volatile int32_t*)err) & kErrCapacity) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  int ntw = hi > lo ? hi - lo : 0;
  int leaf = off[p] + ntw;
  if (leaf >= cap) return;
  int s = p >= n_el;
  double sign = s ? 1.0 : -1.0;
  uint32_t o = vals[p];
  node_c[leaf] = make_double4(x[3 * (int64_t)o], x[3 * (int64_t)o + 1],
                              x[3 * (int64_t)o + 2], -1.0);
  double2* m = node_m + 5 * (int64_t)leaf;
  m[0] = make_double2(sign, 0.0);
  m[1] = make_double2(0.0, 0.0);
  m[2] = make_double2(0.0, 0.0);
  m[3] = make_double2(0.0, 0.0);
  m[4] = make_double2(0.0, 0.0);
  __threadfence();
  const double smax0 = geom[s].smax0;
  int cur = node_parent[leaf];
  int guard = 0;
  while (cur >= 0) {
    if (++guard > kMaxLevel + 2) {
      set_error(err, kErrWalk);
      return;
    }
    int old = atomicAdd(&node_done[cur], 1);
    if (old != node_nchild[cur] - 1) return;
    __threadfence();
    // ---- PSeudoE/PSeudoI for twig `cur` (tree.f90:465-552) ----
    double4 gc = ldcg_d4(&node_c[cur]);
    double ox0 = gc.x, ox1 = gc.y, ox2 = gc.z;
    int end = node_skip[cur];
    if (end > cap) end = cap;
    double qsum = 0.0, X0 = 0.0, X1 = 0.0, X2 = 0.0;
    int c = cur + 1;
    while (c < end) {
      double4 cc = ldcg_d4(&node_c[c]);
      double q = __ldcg(&node_m[5 * (int64_t)c]).x;
      qsum = qsum + q;
      X0 = X0 + q * cc.x;
      X1 = X1 + q * cc.y;
      X2 = X2 + q * cc.z;
      int nx = node_skip[c];
      if (nx <= c) { set_error(err, kErrWalk); return; }
      c = nx;
    }
    X0 = X0 / qsum;
    X1 = X1 / qsum;
    X2 = X2 / qsum;
    double a0 = X0 - ox0, a1 = X1 - ox1, a2 = X2 - ox2;
    double dx = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
    double D0 = 0.0, D1 = 0.0, D2 = 0.0, Q0 = 0.0, Q1 = 0.0, Q2 = 0.0,
           QQ0 = 0.0, QQ1 = 0.0, QQ2 = 0.0;
    c = cur + 1;
    while (c < end) {
      double4 cc = ldcg_d4(&node_c[c]);
      double q = __ldcg(&node_m[5 * (int64_t)c]).x;
      double d0 = cc.x - X0, d1 = cc.y - X1, d2 = cc.z - X2;
      D0 = D0 + q * d0;
      D1 = D1 + q * d1;
      D2 = D2 + q * d2;
      Q0 = Q0 + q * (d0 * d0) / 2.0;
      Q1 = Q1 + q * (d1 * d1) / 2.0;
      Q2 = Q2 + q * (d2 * d2) / 2.0;
      QQ0 = QQ0 + q * d0 * d1;
      QQ1 = QQ1 + q * d1 * d2;
      QQ2 = QQ2 + q * d2 * d0;
      c = node_skip[c];
    }
    // s = MAXVAL(P%lx) at this level: each axis halves exactly per level.
    int lev = node_level[cur];
    double smax = smax0;
    for (int l = 0; l < lev; ++l) smax = smax * 0.5;
    double rcrit = smax / theta + dx;
    node_c[cur] = make_double4(X0, X1, X2, rcrit);
    double2* mm = node_m + 5 * (int64_t)cur;
    mm[0] = make_double2(qsum, D0);
    mm[1] = make_double2(D1, D2);
    mm[2] = make_double2(Q0, Q1);
    mm[3] = make_double2(Q2, QQ0);
    mm[4] = make_double2(QQ1, QQ2);
    __threadfence();
    cur = node_parent[cur];
  }
}

// ------------------------------------------------------------ groups ----
// Target groups of the mixed walk: maximal cells holding at most kGroupMax
// particles, with consecutive small siblings packed together up to kGroupMax.
// Every group is a contiguous sorted range inside one parent cell.  Packing
// is limited to parents at most kGroupSlack + 1 levels above the cloud's
// typical group level (the particle-weighted median level of its maximal
// cells): the sparse octants of a large parent -- escaped electrons around a
// dense core -- would otherwise share one group whose bounding box spans the
// parent and contains the core, and that one warp opens the whole tree.
// Group order is not deterministic (atomic append); the content of every
// group is.
constexpr int kGroupSlack = 3;

// Particle-weighted histogram of the levels of the maximal cells holding at
// most kGroupMax particles, per cloud: glvl[seg * kLevelSlots + level].
__global__ void k_group_levels(const int32_t* __restrict__ bounds, int cap,
                               const int32_t* __restrict__ node_parent,
                               const int8_t* __restrict__ node_level, MixedNodes mx,
                               Ensemble ens, int32_t* glvl) {
  const int m = bounds[2] < cap ? bounds[2] : cap;
  // warp-uniform loop: every lane reaches the collectives of each round
  for (int base = blockIdx.x * blockDim.x; base < m; base += gridDim.x * blockDim.x) {
    const int t = base + threadIdx.x;
    int slot = -1, w = 0;
    if (t < m) {
      const int cnt = mx.count[t];
      const int par = node_parent[t];
      if (cnt <= kGroupMax && (par < 0 || mx.count[par] > kGroupMax)) {
        const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, mx.first[t]) : 0;
        slot = seg * kLevelSlots + node_level[t];
        w = cnt;
      }
    }
    // one atomic per distinct slot per warp
    const unsigned peers = __match_any_sync(0xffffffffu, slot);
    const int sum = __reduce_add_sync(peers, w);
    if (slot >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&glvl[slot], sum);
  }
}

// Per cloud: the lowest level at which siblings may be packed, stored in the
// last slot of the cloud's histogram row (levels stay below kLevelSlots - 1).
__global__ void k_group_cut(int32_t* glvl, int nseg) {
  const int seg = blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= nseg) return;
  int32_t* h = glvl + (int64_t)seg * kLevelSlots;
  int64_t tot = 0;
  for (int l = 0; l < kLevelSlots - 1; ++l) tot += h[l];
  int64_t run = 0;
  int med = 0;
  for (int l = 0; l < kLevelSlots - 1; ++l) {
    run += h[l];
    if (2 * run >= tot) {
      med = l;
      break;
    }
  }
  h[kLevelSlots - 1] = med > kGroupSlack ? med - kGroupSlack : 0;
}

__device__ __forceinline__ void groups_of_node(int t, const int32_t* __restrict__ node_parent,
                                               const int8_t* __restrict__ node_level,
                                               const MixedNodes& mx, const Ensemble& ens,
                                               const int32_t* __restrict__ glvl,
                                               int2* groups, int32_t* n_groups) {
  const int cnt = mx.count[t];
  if (node_parent[t] < 0 && cnt <= kGroupMax) {  // a whole tree fits one group
    int g = atomicAdd(n_groups, 1);
    groups[g] = make_int2(mx.first[t], cnt);
    return;
  }
  if (cnt <= kGroupMax || cnt == 1) return;
  const int seg = ens.nseg > 0 ? seg_of(ens.start, ens.nseg, mx.first[t]) : 0;
  const bool pack = node_level[t] + 1 >= glvl[seg * kLevelSlots + kLevelSlots - 1];
  const int4* kk = reinterpret_cast<const int4*>(mx.kids + 8 * (int64_t)t);
  const int4 k0 = kk[0], k1 = kk[1];
  const int kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
  // runs of consecutive small children are cut into balanced contiguous
  // chunks of at most kGroupMax (a chunk may straddle two children, but it
  // stays inside this cell)
  int run_first = -1, run_cnt = 0;
  auto close_run = [&]() {
    if (run_cnt <= 0) return;
    const int k = (run_cnt + kGroupMax - 1) / kGroupMax;
    const int g = atomicAdd(n_groups, k);
    for (int i = 0; i < k; ++i) {
      const int lo = (int)((int64_t)i * run_cnt / k), hi = (int)((int64_t)(i + 1) * run_cnt / k);
      groups[g + i] = make_int2(run_first + lo, hi - lo);
    }
    run_first = -1;
    run_cnt = 0;
  };
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = kv[j];
    if (c < 0) continue;
    const int cc = mx.count[c];
    // a large child is recursed into by its own thread; below a large
    // parent every small child is a group of its own: both close the run
    if (cc > kGroupMax || !pack) close_run();
    if (cc > kGroupMax) continue;
    if (run_cnt == 0) run_first = mx.first[c];
    run_cnt += cc;
  }
  close_run();
}

__global__ void k_groups(const int32_t* __restrict__ bounds, int cap,
                         const int32_t* __restrict__ node_parent,
                         const int8_t* __restrict__ node_level, MixedNodes mx,
                         Ensemble ens, const int32_t* __restrict__ glvl,
                         int2* groups, int32_t* n_groups) {
  const int m = bounds[2] < cap ? bounds[2] : cap;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x)
    groups_of_node(t, node_parent, node_level, mx, ens, glvl, groups, n_groups);
}

// ------------------------------------------------------------- driver ----
int build_trees(const BuildBuffers& b, const double* x, int n, int n_el,
                double theta, int mode, cudaStream_t st, bool full_records) {
  // mode 0: one tree per species (parity path); mode 1: one combined tree
  const int split = mode == 0 ? n_el : n;
  const int T = 256;
  k_bbox_init<<<1, 32, 0, st>>>(b.bbox, b.err);
  if (n == 0) {
    cudaMemsetAsync(b.bounds, 0, 4 * sizeof(int32_t), st);
    return 1;
  }
  int launches = 1;
  int gb = (n + T - 1) / T;
  int gbb = gb < 4 * 148 ? gb : 4 * 148;
  // an ensemble of clouds only exists on the mixed path
  const Ensemble ens = mode == 1 ? b.ens : Ensemble();
  if (ens.nseg > 0) {
    k_bbox_seg<<<ens.nseg, T, 0, st>>>(x, ens.start, b.bbox, b.err);
    k_geom_seg<<<(ens.nseg + 31) / 32, 32, 0, st>>>(b.bbox, ens.start, ens.nseg, b.geom);
  } else {
    k_bbox<<<gbb, T, 0, st>>>(x, n, split, b.bbox, b.err);
    k_geom<<<1, 32, 0, st>>>(b.bbox, n, split, b.geom);
  }
  const int lsb = mode == 0 ? 0 : 1;
  const int top = ens.nseg > 0 ? ens.top : 1 - lsb;
  const int nlev = ens.nseg > 0 ? ens.nlev : kMaxLevel;
  // full keys into keys_alt, their high words into the two halves of keys
  uint64_t* hi = reinterpret_cast<uint64_t*>(b.keys);
  k_keys<<<gb, T, 0, st>>>(x, n, split, lsb, n_el, b.geom, ens, b.keys_alt, hi, b.vals);
  launches += 3;
  // sort the high 64 bits (8 passes over 12-byte pairs), gather the full
  // keys in that order, then order the rare ties fully;
  // a long tie run switches on the one-block full sort (which exits otherwise)
  launches += radix_sort(hi, b.vals, hi + n, b.vals_alt, n, b.sort_hist, b.scan_partial, st);
  k_gather_keys<<<gb, T, 0, st>>>(b.keys_alt, b.vals, n, b.keys);
  launches += 1;
  cudaMemsetAsync(b.bounds + 4, 0, sizeof(int32_t), st);
  k_tie_fix<<<gb, T, 0, st>>>(b.keys, b.vals, n, b.bounds + 4);
  k_sort_block<<<1, kSbThreads, 0, st>>>(b.keys, b.vals, b.keys_alt, b.vals_alt, n,
                                         b.bounds + 4);
  launches += 2;
  k_common_levels<<<gb, T, 0, st>>>(b.keys, n, top, nlev, b.L, b.err);
  k_counts<<<gb, T, 0, st>>>(b.L, n, b.cnt);
  launches += 2 + exclusive_scan(b.cnt, b.off, n, b.scan_partial, true, st);
  k_bounds<<<1, 32, 0, st>>>(b.off, n, split, b.cap, b.bounds, b.err);
  // per-node passes: a grid of one thread per node for trees of up to 2n
  // nodes (the usual size), striding over the device's node count beyond
  // (the capacity can be many times the tree after a co-located start).
  // Blocks run in about index order, so the atomic appends of k_groups come
  // out in about pre-order: the walk takes target groups in that order, and
  // neighbouring warps then share the cells they open.
  const int64_t per_node = b.cap < 2 * (int64_t)n ? b.cap : 2 * (int64_t)n;
  int gcap = (int)((per_node + T - 1) / T);
  if (gcap < 1) gcap = 1;
  if (mode == 0) {
    k_topology<<<gb, T, 0, st>>>(b.keys, b.vals, b.L, b.off, n, split, lsb, b.geom,
                                 b.cap, b.node_c, b.node_skip, b.node_pt,
                                 b.node_parent, b.node_nchild, b.node_done,
                                 b.node_level, b.mx, ens, b.err);
    k_link_children<<<gcap, T, 0, st>>>(b.node_parent, b.bounds, b.cap,
                                        b.node_nchild, b.mx);
    launches += 3;
  } else {
    // node_nchild serves as the owner array (the combined tree counts no children)
    k_owner<<<gb, T, 0, st>>>(b.off, n, b.cap, b.node_nchild);
    k_topology_mixed<<<gcap, T, 0, st>>>(b.keys, b.vals, b.L, b.off, b.node_nchild, b.bounds,
                                         n, n_el, x, b.geom, b.cap, b.node_c, b.node_pt,
                                         b.node_parent, b.node_done, b.node_level, b.mx, ens);
    k_link_children<<<gcap, T, 0, st>>>(b.node_parent, b.bounds, b.cap, nullptr, b.mx);
    launches += 4;
  }
  if (mode == 0) {
    k_upward<<<gb, T, 0, st>>>(x, b.vals, b.L, b.off, n, split, b.geom, theta,
                               b.cap, b.bounds, b.node_c, b.node_m,
                               b.node_skip, b.node_parent, b.node_nchild,
                               b.node_done, b.node_level, b.err);
    return launches + 1;
  }
  launches += net_moments(b, n, theta, ens, full_records, st);
  // the level lists of the upward pass are free again: a single cloud keeps
  // its group-level histogram there, an ensemble has one row per cloud
  const int nsg = ens.nseg > 0 ? ens.nseg : 1;
  int32_t* glvl = ens.nseg > 0 ? ens.glvl : b.mx.lvl;
  cudaMemsetAsync(glvl, 0, sizeof(int32_t) * kLevelSlots * (size_t)nsg, st);
  k_group_levels<<<gcap, T, 0, st>>>(b.bounds, b.cap, b.node_parent, b.node_level, b.mx,
                                     ens, glvl);
  k_group_cut<<<(nsg + 127) / 128, 128, 0, st>>>(glvl, nsg);
  cudaMemsetAsync(b.mx.n_groups, 0, sizeof(int32_t), st);
  k_groups<<<gcap, T, 0, st>>>(b.bounds, b.cap, b.node_parent, b.node_level, b.mx, ens,
                               glvl, b.mx.groups, b.mx.n_groups);
  launches += 5;
  if (ens.nseg > 0) {
    k_roots<<<(ens.nseg + 31) / 32, 32, 0, st>>>(b.off, ens.start, ens.nseg, ens.roots);
    launches += 1;
  }
  return launches;
}

}  // namespace tg
