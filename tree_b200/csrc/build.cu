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
//   2. replays each particle's path for 21 levels into a 63-bit key (3 bits
//      per level, child digit = bx + 2 by + 4 bz, the reference's bias-1),
//      with the species in bit 63,
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

// ---------------------------------------------------------------- keys ----
// Replays Insert_Tree's descent (tree.f90:132-173 comparisons, 123-126 child
// centres) for 21 levels.
__global__ void k_keys(const double* __restrict__ x, int n, int n_el,
                       const Geom* __restrict__ geom, uint64_t* keys,
                       uint32_t* vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = i >= n_el;
  const Geom& G = geom[s];
  double p[3], c[3], lx[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[k] = x[3 * (int64_t)i + k];
    c[k] = G.c0[k];
    lx[k] = G.lx0[k];
  }
  uint64_t key = 0;
  for (int l = 0; l < kMaxLevel; ++l) {
    uint32_t b = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      bool hi = !(p[k] < c[k]);
      b |= (uint32_t)hi << k;
      c[k] = c[k] + (hi ? 0.25 : -0.25) * lx[k];
      lx[k] = lx[k] * 0.5;
    }
    key = (key << 3) | b;
  }
  keys[i] = key | (s ? kSpeciesBit : 0ull);
  vals[i] = (uint32_t)i;
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
constexpr int kRsIters = 16;                       // items per lane
constexpr int kRsTile = kRsThreads * kRsIters;     // 4096 items per block
constexpr int kRsBins = 256;

int radix_blocks(int n) { return (n + kRsTile - 1) / kRsTile; }

__global__ void k_rs_hist(const uint64_t* __restrict__ keys, int n, int shift,
                          int32_t* hist /* [256][nb] */) {
  __shared__ int32_t h[kRsBins];
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int j = 0; j < kRsIters; ++j) {
    int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kRsBins; b += blockDim.x)
    hist[(int64_t)b * gridDim.x + blockIdx.x] = h[b];
}

// Stable scatter: tile order is warp-major (warp w owns items
// [w*512, w*512+512) of the tile), then iteration, then lane.
__global__ void __launch_bounds__(kRsThreads)
    k_rs_scatter(const uint64_t* __restrict__ keys_in,
                 const uint32_t* __restrict__ vals_in, int n, int shift,
                 const int32_t* __restrict__ offs /* scanned [256][nb] */,
                 uint64_t* __restrict__ keys_out,
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
  uint64_t k[kRsIters];
  uint32_t v[kRsIters];
  int32_t loc[kRsIters];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kRsIters; ++j) {
    int64_t i = wbase + j * 32 + lane;
    bool ok = i < n;
    k[j] = ok ? keys_in[i] : 0ull;
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

// Sorts (keys, vals) in place using the alternate buffers; 8 passes of 8
// bits, so the result ends in the primary buffers.
int radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt,
               uint32_t* vals_alt, int n, int32_t* hist, int32_t* partial,
               cudaStream_t st) {
  if (n <= 1) return 0;
  int launches = 0;
  int nb = radix_blocks(n);
  uint64_t* kin = keys;
  uint32_t* vin = vals;
  uint64_t* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int pass = 0; pass < 8; ++pass) {
    int shift = pass * 8;
    k_rs_hist<<<nb, kRsThreads, 0, st>>>(kin, n, shift, hist);
    launches += 2 + exclusive_scan(hist, hist, kRsBins * nb, partial, false, st);
    k_rs_scatter<<<nb, kRsThreads, 0, st>>>(kin, vin, n, shift, hist, kout,
                                            vout);
    uint64_t* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
  }
  return launches;
}

// ------------------------------------------------------------ topology ----
// L[p] = number of leading levels that sorted keys p and p+1 share (same
// species), else -1.  Identical keys mean the 21-level cap was hit.
__global__ void k_common_levels(const uint64_t* __restrict__ keys, int n,
                                int8_t* L, int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int8_t r = -1;
  if (p + 1 < n) {
    uint64_t a = keys[p], b = keys[p + 1];
    uint64_t x = a ^ b;
    if ((x >> 63) == 0) {
      if (x == 0) {
        set_error(err, kErrDepth);
        r = kMaxLevel;
      } else {
        int lz = __clzll((long long)x);  // >= 1 (species bit equal)
        r = (int8_t)((lz - 1) / 3);
      }
    }
  }
  L[p] = r;
}

__device__ __forceinline__ void lo_hi(const int8_t* __restrict__ L, int p,
                                      int& lo, int& hi) {
  lo = p == 0 ? -1 : (int)L[p - 1];
  hi = (int)L[p];
  if (lo < 0 && hi < 0) hi = 0;  // single-particle species: root + leaf
}

__global__ void k_counts(const int8_t* __restrict__ L, int n, int32_t* cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  cnt[p] = (hi > lo ? hi - lo : 0) + 1;
}

// first q in [lo_i, hi_i) with (keys[q] >> sh) > pre ; keys sorted
__device__ __forceinline__ int upper_prefix(const uint64_t* __restrict__ keys,
                                            int lo_i, int hi_i, int sh,
                                            uint64_t pre) {
  while (lo_i < hi_i) {
    int mid = lo_i + ((hi_i - lo_i) >> 1);
    if ((keys[mid] >> sh) > pre) hi_i = mid;
    else lo_i = mid + 1;
  }
  return lo_i;
}
// first q in [lo_i, hi_i) with (keys[q] >> sh) >= pre
__device__ __forceinline__ int lower_prefix(const uint64_t* __restrict__ keys,
                                            int lo_i, int hi_i, int sh,
                                            uint64_t pre) {
  while (lo_i < hi_i) {
    int mid = lo_i + ((hi_i - lo_i) >> 1);
    if ((keys[mid] >> sh) >= pre) hi_i = mid;
    else lo_i = mid + 1;
  }
  return lo_i;
}

__device__ __forceinline__ int shift_for_level(int d) { return 63 - 3 * d; }

// Index of the twig at level d that contains sorted particle p, given that it
// was opened at an earlier particle (first particle of the level-d prefix).
__device__ __forceinline__ int twig_index_before(
    const uint64_t* __restrict__ keys, const int8_t* __restrict__ L,
    const int32_t* __restrict__ off, int sb, int p, int d) {
  int sh = shift_for_level(d);
  uint64_t pre = keys[p] >> sh;
  int q = lower_prefix(keys, sb, p + 1, sh, pre);
  int lo_q = q == 0 ? -1 : (int)L[q - 1];
  return off[q] + (d - lo_q - 1);
}

// Writes every node in pre-order.  node_c.xyz of twigs receives the
// geometric centre (replayed like k_keys); the upward pass replaces it.
__global__ void k_topology(const uint64_t* __restrict__ keys,
                           const uint32_t* __restrict__ vals,
                           const int8_t* __restrict__ L,
                           const int32_t* __restrict__ off, int n, int n_el,
                           const Geom* __restrict__ geom, int cap,
                           double4* node_c, int32_t* node_skip,
                           int32_t* node_pt, int32_t* node_parent,
                           int32_t* node_nchild, int32_t* node_done,
                           int8_t* node_level, int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo, hi;
  lo_hi(L, p, lo, hi);
  int s = p >= n_el;
  int sb = s ? n_el : 0, se = s ? n : n_el;
  int tree_end = off[se];
  int base = off[p];
  uint64_t key = keys[p];
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
      int sk;
      if (d == 0) {
        sk = tree_end;
      } else {
        int sh = shift_for_level(d);
        int q = upper_prefix(keys, p + 1, se, sh, key >> sh);
        sk = q < se ? off[q] : tree_end;
      }
      node_skip[idx] = sk;
      int par;
      if (d == 0) par = -1;
      else if (d > lo + 1) par = idx - 1;
      else par = twig_index_before(keys, L, off, sb, p, d - 1);
      node_parent[idx] = par;
    }
    // descend one level along this particle's digits
    if (d < kMaxLevel) {
      int dig = (int)((key >> (60 - 3 * d)) & 7);
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
  node_parent[leaf] = ntw > 0 ? leaf - 1
                              : twig_index_before(keys, L, off, sb, p, depth - 1);
}

// Counts children per twig (separate launch so the zeroing in k_topology is
// complete).
__global__ void k_link_children(const int32_t* __restrict__ node_parent,
                                const int32_t* __restrict__ bounds, int cap,
                                int32_t* node_nchild) {
  int m = bounds[2] < cap ? bounds[2] : cap;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int par = node_parent[i];
  if (par >= 0) atomicAdd(&node_nchild[par], 1);
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

// ------------------------------------------------------------- driver ----
int build_trees(const BuildBuffers& b, const double* x, int n, int n_el,
                double theta, cudaStream_t st) {
  const int T = 256;
  k_bbox_init<<<1, 32, 0, st>>>(b.bbox, b.err);
  if (n == 0) {
    cudaMemsetAsync(b.bounds, 0, 4 * sizeof(int32_t), st);
    return 1;
  }
  int launches = 1;
  int gb = (n + T - 1) / T;
  int gbb = gb < 4 * 148 ? gb : 4 * 148;
  k_bbox<<<gbb, T, 0, st>>>(x, n, n_el, b.bbox, b.err);
  k_geom<<<1, 32, 0, st>>>(b.bbox, n, n_el, b.geom);
  k_keys<<<gb, T, 0, st>>>(x, n, n_el, b.geom, b.keys, b.vals);
  launches += 3;
  launches += radix_sort(b.keys, b.vals, b.keys_alt, b.vals_alt, n,
                         b.sort_hist, b.scan_partial, st);
  k_common_levels<<<gb, T, 0, st>>>(b.keys, n, b.L, b.err);
  k_counts<<<gb, T, 0, st>>>(b.L, n, b.cnt);
  launches += 2 + exclusive_scan(b.cnt, b.off, n, b.scan_partial, true, st);
  k_bounds<<<1, 32, 0, st>>>(b.off, n, n_el, b.cap, b.bounds, b.err);
  k_topology<<<gb, T, 0, st>>>(b.keys, b.vals, b.L, b.off, n, n_el, b.geom,
                               b.cap, b.node_c, b.node_skip, b.node_pt,
                               b.node_parent, b.node_nchild, b.node_done,
                               b.node_level, b.err);
  int gcap = (b.cap + T - 1) / T;
  k_link_children<<<gcap, T, 0, st>>>(b.node_parent, b.bounds, b.cap,
                                      b.node_nchild);
  k_upward<<<gb, T, 0, st>>>(x, b.vals, b.L, b.off, n, n_el, b.geom, theta, b.cap, b.bounds, b.node_c, b.node_m,
                             b.node_skip, b.node_parent, b.node_nchild,
                             b.node_done, b.node_level, b.err);
  return launches + 4;
}

}  // namespace tg
