// walk_mixed.h -- warp-group mixed-precision walk (FP32 cell-relative).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "build.h"
#include "internal.cuh"
#include "walk.h"

namespace tg {

struct MixedBuffers {
  int cap = 0;
  int n = 0;
};

inline int mixed_alloc_nodes(MixedBuffers& mb, int cap) {
  mb.cap = cap;
  return 0;
}
inline int mixed_alloc_particles(MixedBuffers& mb, int n) {
  mb.n = n;
  return 0;
}
inline void mixed_free(MixedBuffers&) {}

// Not built yet: flags a walk error so the caller fails loudly.
inline void walk_mixed(MixedBuffers&, const BuildBuffers& b, const double*,
                       int, int, const TreeView&, const WalkParams&, int, int,
                       double*, double2*, uint32_t*, unsigned long long*,
                       int32_t* err, cudaStream_t st) {
  (void)b;
  int32_t bit = kErrWalk;
  cudaMemcpyAsync(err, &bit, sizeof(bit), cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
}

}  // namespace tg
