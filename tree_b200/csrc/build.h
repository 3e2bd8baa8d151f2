// build.h -- device buffers and entry points of the octree build.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "internal.cuh"

namespace tg {

// Node data of the combined tree that the mixed-precision walk reads.
constexpr int kGroupMax = 32;  // targets per warp group
constexpr int kM64 = 19;       // double2 per node of net-charge moments
struct MixedNodes {
  int32_t* kids;     // 8 per node: child index per octant digit, -1 if none
  int32_t* first;    // first sorted particle of the node's range
  int32_t* count;    // particles in the node
  int8_t* digit;     // octant of the node inside its parent
  double2* m64;      // 19 per node: (n, Q) (Dx, Dy) (Dz, q_ion) (Sxx, Syy) (Szz, Sxy) (Syz, Szx) T[10] H[15] 0
  float4* mom;       // 3 per node: (Q, Dx, Dy, Dz) (Sxx, Syy, Szz, Sxy) (Syz, Szx, trS, q_ion)
  float4* mom3;      // 3 per node: third moment T (10) and |T|_F
  float4* mom4;      // 3 per node: 12 components of the trace-free fourth moment H'
  float4* geom;      // per node: (box side s, |centroid - box centre|, n, 0)
  double4* xs;       // per sorted particle: position, w = 1 for ions
  int2* groups;      // target groups (first sorted particle, count)
  int32_t* n_groups; // device count of groups
  int32_t* lvl_list; // per node: twigs grouped by level (upward pass)
  int32_t* lvl;      // kLevelSlots x 3: count, offset, cursor per level
  int32_t* cls;      // net pass: class counts per block of 1024 nodes (class-major),
                     // then their exclusive scan (net_cls_entries(cap) in all)
};

// Entries of MixedNodes::cls for node capacity cap.
inline int net_cls_entries(int cap) { return 2 * 7 * ((cap + 1023) / 1024); }

constexpr int kLevelSlots = 64;  // > deepest twig level

// Independent clouds in one combined forest (mixed path only).  Cloud c holds
// particles [start[c], start[c+1]) of the index space, electrons first up to
// elec_end[c]; its key carries c in the top `top` bits above nlev spatial
// levels, so one sort groups the clouds and its tree is rooted at node
// roots[c].  nseg = 0: a single cloud with the classic layout.
struct Ensemble {
  int nseg = 0;
  int top = 0;
  int nlev = kMaxLevel;
  const int32_t* start = nullptr;     // device, nseg + 1
  const int32_t* elec_end = nullptr;  // device, nseg
  int32_t* roots = nullptr;           // device, nseg
  int32_t* glvl = nullptr;            // device, nseg x kLevelSlots (target groups)
};

struct BuildBuffers {
  // particle-indexed (n)
  key128* keys;
  key128* keys_alt;
  uint32_t* vals;       // sorted position -> global particle index
  uint32_t* vals_alt;
  int8_t* L;            // common levels with the next sorted key
  int32_t* cnt;         // nodes emitted per sorted particle
  int32_t* off;         // exclusive scan of cnt (n+1)
  int32_t* sort_hist;   // 256 * radix blocks
  int32_t* scan_partial;
  // node-indexed (cap)
  int cap;
  double4* node_c;
  double2* node_m;
  int32_t* node_skip;
  int32_t* node_pt;
  int32_t* node_parent;
  int32_t* node_nchild;
  int32_t* node_done;
  int8_t* node_level;
  // small
  uint64_t* bbox;       // 6 per segment (>= 2 segments)
  Geom* geom;           // per segment (>= 2)
  int32_t* bounds;      // 5: 0, M_e, M (clamped to cap), M (untruncated), long-tie flag
  int32_t* err;
  MixedNodes mx;
  Ensemble ens;
};

// Largest c with start[c] <= i (start[0] = 0, nseg entries searched).
__device__ __forceinline__ int seg_of(const int32_t* __restrict__ start, int nseg,
                                      int i) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(&start[mid]) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Sorted particle p's common levels with its neighbours: lo with p - 1, hi
// with p + 1 (-1 where the species ends).
__device__ __forceinline__ void lo_hi(const int8_t* __restrict__ L, int p,
                                      int& lo, int& hi) {
  lo = p == 0 ? -1 : (int)L[p - 1];
  hi = (int)L[p];
  if (lo < 0 && hi < 0) hi = 0;  // single-particle species: root + leaf
}

int radix_blocks(int n);
int scan_partials_needed(int n);
int exclusive_scan(const int32_t* in, int32_t* out, int n, int32_t* partial,
                   bool write_total, cudaStream_t st);
// Stable LSD radix sort of (keys, vals) by all bytes of the key (8 passes for
// uint64_t keys, 16 for key128); the result ends in the primary buffers.
// first_byte > 0 skips the low bytes (an even number of passes must remain).
template <class K>
int radix_sort(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int n,
               int32_t* hist, int32_t* partial, cudaStream_t st, int first_byte = 0);
// Builds the trees for positions x (AoS, electrons first).  mode 0: one tree
// per species with the reference's one-level moments (parity path); mode 1:
// one combined tree with net-charge moments and target groups (mixed path).
// full_records (mode 1): write every twig's FP64 moment record (m64), which
// only the learned criterion's sampler and the debug dump read; otherwise only
// the records that the build itself needs are written.
int build_trees(const BuildBuffers& b, const double* x, int n, int n_el,
                double theta, int mode, cudaStream_t st, bool full_records = false);
// The net-charge moments of the combined tree (mode 1) once its topology and
// child tables exist.
int net_moments(const BuildBuffers& b, int n, double theta, const Ensemble& ens,
                bool full_records, cudaStream_t st);

}  // namespace tg
