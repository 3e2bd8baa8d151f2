// walk_mixed.h -- warp-group mixed-precision walk (FP32 cell-relative).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "build.h"
#include "internal.cuh"
#include "mlp.cuh"
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
  float4* mom3 = nullptr;
  float4* mom4 = nullptr;
  float4* geom = nullptr;
  float2* mac_k = nullptr;     // learned MAC: the cell's pre-filter record
  double4* xs = nullptr;
  int2* groups = nullptr;
  int32_t* lvl_list = nullptr; // per node: twigs by level (upward pass)
  int32_t* lvl = nullptr;      // per level: count, offset, cursor
  int32_t* cls = nullptr;      // net pass: class counts per node block, then their scan
  int32_t* stack = nullptr;    // per resident warp: kStackCap node indices
  int32_t* control = nullptr;  // [0] group cursor, [1] max stack depth, [2] groups
  int grid_warps = 0;
};

// Tunables of the walk (picked by tree_b200/tune.py; defaults below).
struct MixedTuning {
  int bucket = 8;          // twigs with <= bucket particles are summed directly
  int blocks_per_sm = 4;   // persistent grid: SMs x blocks_per_sm blocks
  int order = 3;           // far-field order: 2 quadrupole, 3 octupole, 4 hexadecapole
  // accepted cells far from a target group are summed into the group's local
  // expansion (local.cuh) when (group half-diagonal) / (distance from the
  // group centre to the cell's centroid) <= loc_eps; 0 = every accepted cell
  // is evaluated at every target.  0.08 keeps the force error of the
  // N = 1M cloud unchanged within 2 % (rms) and shortens the walk by 16 %.
  float loc_eps = 0.08f;
};

// Learned acceptance: a cell the fixed-theta test opens, with s/(d - dx) <=
// rho_hi, is accepted when the predicted error 10^y * n/d^2 (units of e,
// Coulomb constant dropped) is at most eta * min over the group of
// |F_prev| / eps.
struct LearnedMac {
  const MlpPacked* packed = nullptr;  // device
  const float* fmin = nullptr;        // device, 16: training range
  const float* fmax = nullptr;        // device, 16
  const float* margins = nullptr;     // device, 7: m_lo, m_hi, pre-filter c0..c4
  const double* f_prev = nullptr;     // device forces of the previous step
  float eta = 1e-5f;
  float rho_lo = 0.2f, rho_hi = 0.9f;
  float lam_ei = 0.f;
};

int mixed_alloc_nodes(MixedBuffers& mb, int cap);
int mixed_alloc_particles(MixedBuffers& mb, int n);
void mixed_free(MixedBuffers& mb);
MixedNodes mixed_nodes(const MixedBuffers& mb);

// Forces on every particle from both trees.  Returns kernels launched.
int walk_mixed(MixedBuffers& mb, const BuildBuffers& b, const double* x,
               int n, int n_el, const TreeView& tv, const WalkParams& wp,
               const MixedTuning& tune, const LearnedMac* learned,
               const Ensemble& ens, const float4* cloud_pk,
               double* f, double2* epot_part,
               uint32_t* rdf, unsigned long long* counters, int32_t* err,
               cudaStream_t st);

}  // namespace tg
