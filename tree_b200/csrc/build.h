// build.h -- device buffers and entry points of the octree build.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "internal.cuh"

namespace tg {

struct BuildBuffers {
  // particle-indexed (n)
  uint64_t* keys;
  uint64_t* keys_alt;
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
  uint64_t* bbox;       // 12
  Geom* geom;           // 2
  int32_t* bounds;      // 4: 0, M_e, M (clamped to cap), M (untruncated)
  int32_t* err;
};

int radix_blocks(int n);
int scan_partials_needed(int n);
int exclusive_scan(const int32_t* in, int32_t* out, int n, int32_t* partial,
                   bool write_total, cudaStream_t st);
int radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt,
                uint32_t* vals_alt, int n, int32_t* hist, int32_t* partial,
                cudaStream_t st);
// Builds both species trees for positions x (AoS, electrons first).
int build_trees(const BuildBuffers& b, const double* x, int n, int n_el,
                 double theta, cudaStream_t st);

}  // namespace tg
