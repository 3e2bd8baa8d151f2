// kdk.h -- integrator and diagnostic reductions.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tg {

int kdk_partials_needed(int n);
// VVerletNotemp1 for all particles (electrons [0,n_el) use xm_e; with a
// per-particle ion flag, as in an ensemble of clouds, the flag decides).
void kick_drift(double* x, double* v, const double* f, int n, int n_el,
                const uint8_t* ion, double dt, double xm_e, double xm_i,
                cudaStream_t st);
// VVerletNotemp2 (+ next VVerletNotemp1 when drift).  When sample, out4 gets
// (mv2_el, rad_el, mv2_ion, rad_ion) of the state after the second kick.
void kick2(double* x, double* v, const double* f, int n, int n_el,
           const uint8_t* ion, double dt, double xm_e, double xm_i, bool sample,
           bool drift, double* partial, double* out4, cudaStream_t st);
// Per-cloud (Epot_e, Epot_i, mv2_el, mv2_ion, rad_el, rad_ion) of an ensemble.
void cloud_sums(const double* x, const double* v, const double2* ep,
                const int32_t* start, const int32_t* elec_end, int nseg,
                double xm_e, double xm_i, double* out, cudaStream_t st);
// out4 = (Epot_e, Epot_i, 0, 0); counters[4..7] += counters[0..3] (the
// walk's per-step interaction counts into running totals) when not NULL.
void epot_sum(const double2* ep, int n, double* partial, double* out4,
              unsigned long long* counters, cudaStream_t st);
// Appends (Epot_e, Epot_i, mv2_el, mv2_ion, rad_el, rad_ion) from diag[8]
// to series[*count] while *count < cap (one record per sample step).
void sample_append(const double* diag, double* series, int32_t* count, int cap,
                   cudaStream_t st);
// acc64[i] += bins32[i] for 2 * kRdfBins bins (running RDF sums of a run).
void rdf_fold(const uint32_t* bins32, unsigned long long* acc64, cudaStream_t st);

}  // namespace tg
