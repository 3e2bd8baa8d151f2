// walk_mixed.h -- warp-group mixed-precision walk (FP32 cell-relative).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "build.h"
#include "internal.cuh"
#include "walk.h"

namespace tg {

struct MixedBuffers {
  int cap = 0;       // node capacity of the arrays below
  int n = 0;         // particles
  int32_t* kids = nullptr;
  int32_t* first = nullptr;
  int32_t* count = nullptr;
  int8_t* digit = nullptr;
  double2* m64 = nullptr;
  float4* mom = nullptr;
  double4* xs = nullptr;
  int2* groups = nullptr;
  int32_t* stack = nullptr;    // per resident warp: kStackCap node indices
  int32_t* control = nullptr;  // [0] group cursor, [1] max stack depth, [2] groups
  int grid_warps = 0;
};

// Tunables of the walk (picked by tree_b200/tune.py; defaults below).
struct MixedTuning {
  int bucket = 4;          // twigs with <= bucket particles are summed directly
  int blocks_per_sm = 4;   // persistent grid: SMs x blocks_per_sm blocks
};

int mixed_alloc_nodes(MixedBuffers& mb, int cap);
int mixed_alloc_particles(MixedBuffers& mb, int n);
void mixed_free(MixedBuffers& mb);
MixedNodes mixed_nodes(const MixedBuffers& mb);

// Forces on every particle from both trees.  Returns kernels launched.
int walk_mixed(MixedBuffers& mb, const BuildBuffers& b, const double* x,
               int n, int n_el, const TreeView& tv, const WalkParams& wp,
               const MixedTuning& tune, double* f, double2* epot_part,
               uint32_t* rdf, unsigned long long* counters, int32_t* err,
               cudaStream_t st);

}  // namespace tg
