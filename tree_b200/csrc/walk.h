// walk.h -- tree walk entry points.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "internal.cuh"

namespace tg {

struct WalkParams {
  int physics;     // 0 REF, 1 KELBG
  double theta;
  double rs;       // REF e-i screening length
  double lam_ee, lam_ei, lam_ii;
  double dx_ei, dx_ii;
};

// FP64 per-target walk (parity path).  rdf may be null (2 x 10001 u32).
// counters[0] += accepted cells, counters[1] += leaf pairs.
void walk64(const double* x, int n, int n_el, const uint32_t* order,
            const TreeView& tv, const WalkParams& wp, double* f,
            double2* epot_part, uint32_t* rdf, unsigned long long* counters,
            int32_t* err, cudaStream_t st);

}  // namespace tg
