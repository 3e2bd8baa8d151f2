// direct.h -- FP64 direct-sum judge.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "walk.h"

namespace tg {

// Source chunks used for nt targets over n sources (partial has nchunks*nt).
int direct_chunks(int n, int nt);
// f (3*nt) and epot (nt, 0.5*sum V) for targets (global particle indices).
// Returns the number of kernels launched.
int direct_sum(const double* x, int n, int n_el, const int64_t* targets,
               int nt, const WalkParams& wp, int nchunks, double4* partial,
               double* f, double* epot, cudaStream_t st);

}  // namespace tg
