// walk64.cu -- FP64 per-target tree walk (parity path; compiled -fmad=false).
//
// Each thread owns one target (targets in Morton order, so a warp's targets
// are spatial neighbours) and walks the electron tree, then the ion tree, in
// pre-order with subtree-skip links.  Pre-order with children 1..8 is the
// order of the recursive Search_Tree_ee/_ie/_ei/_ii (tree.f90:721-1133), so
// every target sees the same accepted cells and leaves in the same order as
// the reference and sums them in that order: forces agree bit-for-bit except
// where the device exp() differs from the host's by an ulp.
#include "internal.cuh"
#include "pair64.cuh"
#include "walk.h"

namespace tg {

// Far field of tree.f90:744-779 (identical in the four walks).
__device__ __forceinline__ void m2p64(const double2* __restrict__ mm,
                                      double xr0, double xr1, double xr2,
                                      double r2, double r, double ff,
                                      double& f0, double& f1, double& f2,
                                      double& ep) {
  double2 m0 = __ldg(mm + 0), m1 = __ldg(mm + 1), m2 = __ldg(mm + 2),
          m3 = __ldg(mm + 3), m4 = __ldg(mm + 4);
  const double qeff = m0.x, PD0 = m0.y, PD1 = m1.x, PD2 = m1.y;
  const double PQ0 = m2.x, PQ1 = m2.y, PQ2 = m3.x, PQQ0 = m3.y, PQQ1 = m4.x,
               PQQ2 = m4.y;
  double R3 = r2 * r;
  double R5 = R3 * r2;
  double R7 = R5 * r2;
  double D0 = -1.0 / R3 + 3.0 * (xr0 * xr0) / R5;
  double D1 = -1.0 / R3 + 3.0 * (xr1 * xr1) / R5;
  double D2 = -1.0 / R3 + 3.0 * (xr2 * xr2) / R5;
  double D3 = 3.0 * xr0 * xr1 / R5;
  double D4 = 3.0 * xr1 * xr2 / R5;
  double D5 = 3.0 * xr2 * xr0 / R5;
  double Q0 = 15.0 * ((xr0 * xr0) * xr0) / R7 - 9.0 * xr0 / R5;
  double Q1 = 15.0 * ((xr1 * xr1) * xr1) / R7 - 9.0 * xr1 / R5;
  double Q2 = 15.0 * ((xr2 * xr2) * xr2) / R7 - 9.0 * xr2 / R5;
  double Q3 = 15.0 * (xr0 * xr0) * xr1 / R7 - 3.0 * xr1 / R5;
  double Q4 = 15.0 * (xr0 * xr0) * xr2 / R7 - 3.0 * xr2 / R5;
  double Q5 = 15.0 * (xr1 * xr1) * xr0 / R7 - 3.0 * xr0 / R5;
  double Q6 = 15.0 * (xr1 * xr1) * xr2 / R7 - 3.0 * xr2 / R5;
  double Q7 = 15.0 * (xr2 * xr2) * xr0 / R7 - 3.0 * xr0 / R5;
  double Q8 = 15.0 * (xr2 * xr2) * xr1 / R7 - 3.0 * xr1 / R5;
  double Q9 = 15.0 * xr0 * xr1 * xr2 / R7;
  ep = ep + 0.5 * ff *
                (qeff / r + (PD0 * xr0 + PD1 * xr1 + PD2 * xr2) / R3 +
                 PQ0 * D0 + PQ1 * D1 + PQ2 * D2 + PQQ0 * D3 + PQQ1 * D4 +
                 PQQ2 * D5);
  f0 = f0 + ff * (qeff * xr0 / R3 + D0 * PD0 + D3 * PD1 + D5 * PD2 +
                  Q0 * PQ0 + Q5 * PQ1 + Q7 * PQ2 + Q3 * PQQ0 + Q4 * PQQ2 +
                  Q9 * PQQ1);
  f1 = f1 + ff * (qeff * xr1 / R3 + D3 * PD0 + D1 * PD1 + D4 * PD2 +
                  Q3 * PQ0 + Q1 * PQ1 + Q8 * PQ2 + Q5 * PQQ0 + Q9 * PQQ2 +
                  Q6 * PQQ1);
  f2 = f2 + ff * (qeff * xr2 / R3 + D5 * PD0 + D4 * PD1 + D2 * PD2 +
                  Q4 * PQ0 + Q6 * PQ1 + Q2 * PQ2 + Q9 * PQQ0 + Q7 * PQQ2 +
                  Q8 * PQQ1);
}

__device__ __forceinline__ void rdf_add(uint32_t* hist, double r,
                                        double dxbin) {
  // id = INT(r/dx)+1 ; counted when 0 < id <= Ndist+1 (tree.f90:916-919)
  double t = r / dxbin;
  if (!(t < (double)kRdfBins)) return;
  int id = (int)t;
  if (id >= 0) atomicAdd(&hist[id], 1u);
}

template <int PHYS, bool RDF>
__global__ void __launch_bounds__(128)
    k_walk64(const double* __restrict__ x, int n, int n_el,
             const uint32_t* __restrict__ order, TreeView tv, WalkParams wp,
             double* __restrict__ f, double2* __restrict__ epot_part,
             uint32_t* __restrict__ rdf, unsigned long long* counters,
             int32_t* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = p < n;
  if (*((volatile int32_t*)err) & (kErrCapacity | kErrDepth | kErrNonFinite))
    return;
  int64_t o = active ? (int64_t)order[p] : 0;
  int tsp = o >= n_el;  // target species: 0 electron, 1 ion
  double xt0 = 0, xt1 = 0, xt2 = 0;
  if (active) {
    xt0 = x[3 * o];
    xt1 = x[3 * o + 1];
    xt2 = x[3 * o + 2];
  }
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  double ep_tree[2] = {0.0, 0.0};
  uint32_t nm2p = 0, np2p = 0;
  const int32_t* bnd = tv.tree_bounds;
  for (int ssp = 0; ssp < 2 && active; ++ssp) {
    int node = bnd[ssp], end = bnd[ssp + 1];
    bool same = ssp == tsp;
    // ff for accepted cells: -eps for electron targets, +eps for ions
    const double ffc = tsp == 0 ? -1.0 * kEps : kEps;
    double ep = 0.0;
    while (node < end) {
      double4 c = ldg_d4(&tv.node_c[node]);
      double xr0 = xt0 - c.x, xr1 = xt1 - c.y, xr2 = xt2 - c.z;
      double r2 = xr0 * xr0 + xr1 * xr1 + xr2 * xr2;
      if (c.w < 0.0) {
        // ---------------- leaf ----------------
        bool self = PHYS == 1 && same && __ldg(&tv.node_pt[node]) == (int)o;
        double r = 0.0;
        if (leaf_pair64<PHYS>(xr0, xr1, xr2, r2, same, tsp, self, wp, f0, f1,
                              f2, ep, r)) {
          ++np2p;
          if (RDF) {
            if (!same) rdf_add(rdf, r, wp.dx_ei);
            else if (tsp == 1 && (PHYS == 0 || r2 > 0.0))
              rdf_add(rdf + kRdfBins, r, wp.dx_ii);
          }
        }
        ++node;
      } else {
        // ---------------- twig: MAC (tree.f90:736-743) ----------------
        double r = sqrt(r2);
        if (c.w < r) {
          ++nm2p;
          m2p64(tv.node_m + 5 * (int64_t)node, xr0, xr1, xr2, r2, r, ffc, f0,
                f1, f2, ep);
          int nx = __ldg(&tv.node_skip[node]);
          if (nx <= node) {
            set_error(err, kErrWalk);
            break;
          }
          node = nx;
        } else {
          ++node;
        }
      }
    }
    ep_tree[ssp] = ep;
  }
  if (active) {
    f[3 * o] = f0;
    f[3 * o + 1] = f1;
    f[3 * o + 2] = f2;
    // Epot_e = ee + ie + ei ; Epot_i = ii (tree.f90:674-715)
    double ee = tsp == 0 ? ep_tree[0] + ep_tree[1] : ep_tree[0];
    double ii = tsp == 0 ? 0.0 : ep_tree[1];
    epot_part[o] = make_double2(ee, ii);
  }
  // interaction counters
  unsigned long long a = nm2p, b = np2p;
  for (int s = 16; s > 0; s >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, s);
    b += __shfl_xor_sync(0xffffffffu, b, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[0], a);
    atomicAdd(&counters[1], b);
  }
}

void walk64(const double* x, int n, int n_el, const uint32_t* order,
            const TreeView& tv, const WalkParams& wp, double* f,
            double2* epot_part, uint32_t* rdf, unsigned long long* counters,
            int32_t* err, cudaStream_t st) {
  if (n == 0) return;
  const int T = 128;
  int g = (n + T - 1) / T;
  bool r = rdf != nullptr;
  if (wp.physics == 0) {
    if (r) k_walk64<0, true><<<g, T, 0, st>>>(x, n, n_el, order, tv, wp, f, epot_part, rdf, counters, err);
    else k_walk64<0, false><<<g, T, 0, st>>>(x, n, n_el, order, tv, wp, f, epot_part, rdf, counters, err);
  } else {
    if (r) k_walk64<1, true><<<g, T, 0, st>>>(x, n, n_el, order, tv, wp, f, epot_part, rdf, counters, err);
    else k_walk64<1, false><<<g, T, 0, st>>>(x, n, n_el, order, tv, wp, f, epot_part, rdf, counters, err);
  }
}

}  // namespace tg
