// internal.cuh -- device-side data layout shared by the kernels of the force
// path.  Nothing here is part of the C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tg {

constexpr double kEps = 0.0014399835661145824;  // data.f90:40 (eV*um)
constexpr int kRdfBins = 10001;                  // Ndist+1 (data.f90:38)
constexpr int kMaxLevel = 42;                    // 3 bits per level in 126 bits

// Particle path keys: 42 levels of 3 bits in an unsigned 128-bit integer.
typedef unsigned __int128 key128;

// error flag bits (device word, read by the host after a call)
enum : int32_t {
  kErrDepth = 1,
  kErrNonFinite = 2,
  kErrCapacity = 4,
  kErrWalk = 8,
};

// Both species share one particle index space: electrons [0, n_el), ions
// [n_el, n).  Positions, velocities, forces are AoS double xyz.
// Both trees share one node index space in pre-order (children visited in
// the reference's order 1..8): electron tree [0, M_e), ion tree [M_e, M).
struct TreeView {
  const double4* __restrict__ node_c;  // (centre xyz, rcrit); rcrit<0: leaf
  const double2* __restrict__ node_m;  // 5 x double2 per node: qeff,D0 | D1,D2
                                       // | Q0,Q1 | Q2,QQ0 | QQ1,QQ2
  const int32_t* __restrict__ node_skip;  // pre-order index past subtree
  const int32_t* __restrict__ node_pt;    // leaf: particle index (global)
  const int32_t* __restrict__ tree_bounds;  // [0]=0, [1]=M_e, [2]=M
};

struct Geom {       // root box of one species (BuildLocalTree tree.f90:52-63)
  double c0[3];     // (max+min)/2
  double lx0[3];    // max-min
  double smax0;     // MAXVAL(lx0)
  int32_t n;        // particles in this species
  int32_t first;    // first global particle index of this species
};

// Order-preserving map double -> uint64 so atomicMin/atomicMax give exact
// min/max of doubles.
__device__ __forceinline__ uint64_t ord_from_double(double d) {
  uint64_t u = (uint64_t)__double_as_longlong(d);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double double_from_ord(uint64_t o) {
  uint64_t u = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
  union { uint64_t u; double d; } cv;
  cv.u = u;
  return cv.d;
}

// L2-coherent (L1-bypassing) load of a double4 written by another block.
__device__ __forceinline__ double4 ldcg_d4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Read-only-path load of a double4 (two 16-byte loads).
__device__ __forceinline__ double4 ldg_d4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ void set_error(int32_t* flag, int32_t bit) {
  atomicOr(flag, bit);
}

}  // namespace tg
