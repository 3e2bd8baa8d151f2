/* tree_gpu.h -- C ABI of the B200 force path for TREE (hpjeonGIT/TREE).
 *
 * The reference computes forces in SUBROUTINE Force(NS, qel, qion, param,
 * ttime) (main.f90:506-701), an internal procedure of PROGRAM OCTREE_HYBRID
 * that builds one octree per species (tree.f90:39-100), computes one-level
 * multipole moments (tree.f90:450-659) and walks both trees for every target
 * (tree.f90:662-1133).  Velocity Verlet is VVerletNotemp1/2 (vverlet.f90:9-112).
 * This header is the drop-in boundary that replaces those calls: plain C
 * types, caller-owned host buffers, library-owned device memory, int status.
 *
 * Arrays of positions/velocities/forces are AoS xyz triples of double
 * (x0,y0,z0,x1,...), the layout of TYPE(GS) (data.f90:54-56) after the
 * Fortran caller packs TYPE(PT)%xx into a REAL(C_DOUBLE) array.
 *
 * Threading: one handle belongs to one host thread and one CUDA stream; calls
 * on a handle are not reentrant.
 */
#ifndef TREE_GPU_H
#define TREE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (0 = ok) */
#define TREE_GPU_OK 0
#define TREE_GPU_ERR_ARG -1        /* bad argument / size */
#define TREE_GPU_ERR_DEPTH -2      /* two same-species particles share the
                                      deepest (42-level) cell; the reference
                                      recurses forever here (tree.f90:128-273) */
#define TREE_GPU_ERR_NONFINITE -3  /* NaN/Inf position */
#define TREE_GPU_ERR_CAPACITY -4   /* internal node capacity exceeded */
#define TREE_GPU_ERR_CUDA -5       /* CUDA runtime error (see last_error) */
#define TREE_GPU_ERR_WALK -6       /* walk guard tripped (corrupt tree) */
#define TREE_GPU_ERR_STATE -7      /* call order (e.g. step before set_state) */

/* physics: which pair laws the leaves use */
#define TREE_GPU_PHYS_REF 0    /* reference laws: Coulomb e-e/i-i with the
                                  r^2 > 0.01 um^2 cutoff (tree.f90:806,1115),
                                  exp-screened e-i "Kelbg" with length rs
                                  (tree.f90:905-913) */
#define TREE_GPU_PHYS_KELBG 1  /* erf-Kelbg for every pair,
                                  lambda_ij = hbar/sqrt(2 mu_ij k T_e) */

/* precision / walk form */
#define TREE_GPU_PREC_FP64 0   /* per-target walk in FP64, the reference's
                                  visiting order (parity path) */
#define TREE_GPU_PREC_MIXED 1  /* warp-group walk, FP32 cell-relative
                                  arithmetic, compensated sums */

/* multipole acceptance criterion */
#define TREE_GPU_MAC_FIXED 0   /* s/theta + dx < r (tree.f90:743) */
#define TREE_GPU_MAC_LEARNED 1 /* learned acceptance, fixed-theta fallback */

#define TREE_GPU_RDF_BINS 10001 /* Ndist + 1 (data.f90:38) */

typedef struct tree_gpu_params {
  double theta;    /* param%sd_ratio (opening criterion) */
  double rs;       /* param%rs, reference e-i screening length (um) */
  double te;       /* electron temperature for lambda_ij (K) */
  double xm_el;    /* param%xm(1), amu */
  double xm_ion;   /* param%xm(2), amu */
  double dx_ei;    /* NS%dx_ei, RDF bin width (um) */
  double dx_ii;    /* NS%dx_ii */
  int32_t physics;   /* TREE_GPU_PHYS_* */
  int32_t precision; /* TREE_GPU_PREC_* */
  int32_t mac;       /* TREE_GPU_MAC_* */
  int32_t group;     /* reserved, 0 (target groups of the mixed walk are
                        maximal cells of at most 32 particles) */
} tree_gpu_params;

typedef struct tree_gpu_diag {
  double epot_e;   /* sys%Epot_e: ee + ie + ei potential energy (eV) */
  double epot_i;   /* sys%Epot_i: ii */
  double mv2_el;   /* sys%mv2el = sum m v^2 (vverlet.f90:86-88) */
  double mv2_ion;  /* sys%mv2ion */
  double rad_el;   /* sys%Te_rad = sum m (x.v)^2/|x|^2 (vverlet.f90:89-91) */
  double rad_ion;  /* sys%Ti_rad */
  int64_t steps_done;
} tree_gpu_diag;

typedef struct tree_gpu_timing {
  double ms_build;   /* bbox + keys + sort + topology + upward pass */
  double ms_walk;    /* tree walk */
  double ms_kdk;     /* kick-drift-kick */
  double ms_total;
  int64_t n_m2p;     /* accepted cells (far-field evaluations), last call */
  int64_t n_p2p;     /* leaf pair evaluations, last call */
  int64_t n_nodes;   /* nodes of both trees, last build */
  int64_t calls;
  int64_t launches;  /* kernels this library launched (cumulative) */
  int64_t n_mac_net;       /* cells the learned MAC evaluated, last call */
  int64_t n_mac_fallback;  /* of those, outside the training range (fixed theta) */
  int64_t n_m2p_total;     /* accepted cells summed over every walk of the handle */
  int64_t n_p2p_total;     /* pair evaluations summed over every walk */
  int64_t n_mac_net_total; /* learned-MAC evaluations summed over every walk */
  int64_t n_local;         /* cells summed into target groups' local expansions, last call */
  int64_t n_local_total;   /* the same, summed over every walk */
} tree_gpu_timing;

typedef struct tree_gpu_handle tree_gpu_handle;

/* Creates a handle for n_el electrons and n_ion ions on the current CUDA
 * device.  Replaces the set-up that Init (main.f90:196-426) and the automatic
 * arrays of Force (main.f90:521-522) did.  */
int tree_gpu_create(const tree_gpu_params* params, int64_t n_el,
                    int64_t n_ion, tree_gpu_handle** out);

/* Changes the parameters (theta, physics, precision, ...) of a handle. */
int tree_gpu_set_params(tree_gpu_handle* h, const tree_gpu_params* params);

/* Force-only drop-in for CALL Force(NS, qel, qion, param, ttime)
 * (main.f90:130, 777, 821).  In: x_el (3*n_el), x_ion (3*n_ion).  Out:
 * f_el, f_ion overwritten (the local part zeroes them, tree.f90:675-680);
 * *epot_e, *epot_i overwritten (sys%Epot_e/_i); rdf_ei, rdf_ii (10001 bins
 * each, may be NULL) are ACCUMULATED like NS%RDF_ei/_ii.  Host buffers; the
 * copies happen inside the call, which returns after the stream synchronises. */
int tree_gpu_force(tree_gpu_handle* h, const double* x_el, const double* x_ion,
                   double* f_el, double* f_ion, double* epot_e,
                   double* epot_i, int64_t* rdf_ei, int64_t* rdf_ii);

/* Loads positions and velocities (host) into the device-resident state and
 * computes the initial forces (what Vinit/Vinit_REST do, main.f90:777/821). */
int tree_gpu_set_state(tree_gpu_handle* h, const double* x_el,
                       const double* v_el, const double* x_ion,
                       const double* v_ion);

/* Loads a full particle state (positions, velocities AND forces, e.g. from a
 * restart or from the caller's own previous step) without computing forces;
 * the next tree_gpu_step starts from it.  Counterpart of the state TYPE(PT)
 * carries between steps (data.f90:47-50). */
int tree_gpu_load_state(tree_gpu_handle* h, const double* x_el,
                        const double* v_el, const double* f_el,
                        const double* x_ion, const double* v_ion,
                        const double* f_ion);

/* Step drop-in for the loop body main.f90:125-131 + VVerletNotemp2: nsteps x
 * (VVerletNotemp1 -> Force -> VVerletNotemp2) on the device with no host
 * traffic.  Kinetic sums are sampled on the last step; `out` may be NULL.
 * Each step body is replayed as a CUDA graph (tree_gpu_set_graphs). */
int tree_gpu_step(tree_gpu_handle* h, double dt, int32_t nsteps,
                  tree_gpu_diag* out);

/* One TEMPORAL sample (sample.f90:55-96 before its unit conversions): the
 * sums VVerletNotemp2 forms on sample steps (vverlet.f90:81-106) and the
 * potential energies of that step's Force. */
typedef struct tree_gpu_sample {
  int64_t nloop;   /* ttime%Nloop of the sample step */
  double epot_e;   /* sys%Epot_e */
  double epot_i;   /* sys%Epot_i */
  double mv2_el;   /* sys%mv2el */
  double mv2_ion;  /* sys%mv2ion */
  double rad_el;   /* sys%Te_rad (sum m (x.v)^2/|x|^2) */
  double rad_ion;  /* sys%Ti_rad */
} tree_gpu_sample;

/* The step loop main.f90:123-160 for nsteps steps with the reference's
 * cadence.  Steps are numbered by Nloop, which tree_gpu_set_state and
 * tree_gpu_load_state reset to 0 (main.f90:113); every step with
 * Nloop % nsamp == 0 (nsamp > 0) forms the kinetic sums and writes one record
 * to series[] (at most series_cap; *n_series = records written), all on the
 * device.  rdf_ei / rdf_ii (kRdfBins = 10001 entries each, either may be
 * NULL) accumulate the near-field pair counts of EVERY step, as NS%RDF_ei /
 * NS%RDF_ii do in Force (tree.f90:918, 1126); the caller dumps and resets
 * them as RDF (sample.f90:5-50) does every Ndump steps.  The FP64 path bins
 * the reference's leaf pairs by their FP64 distance; the mixed path bins the
 * pairs it sums directly by their FP32 distance (within ~1e-6 relative, so a
 * pair that close to a bin edge may fall in the neighbouring bin). */
int tree_gpu_run(tree_gpu_handle* h, double dt, int32_t nsteps, int32_t nsamp,
                 tree_gpu_sample* series, int32_t series_cap, int32_t* n_series,
                 int64_t* rdf_ei, int64_t* rdf_ii);

/* Replays each step body as a CUDA graph (enable != 0, the default) or
 * enqueues its kernels one by one (enable = 0; per-step phase timings). */
int tree_gpu_set_graphs(tree_gpu_handle* h, int32_t enable);

/* Current Nloop of the device-resident state. */
int tree_gpu_get_nloop(tree_gpu_handle* h, int64_t* nloop);

/* Copies the device-resident state to host buffers (any may be NULL), for
 * Restart/RDF/TEMPORAL steps (print.f90:5-109, sample.f90). */
int tree_gpu_get_state(tree_gpu_handle* h, double* x_el, double* v_el,
                       double* f_el, double* x_ion, double* v_ion,
                       double* f_ion);

/* FP64 O(N^2) direct sum (the accuracy judge): forces on the listed targets
 * from every particle at the current device positions, with the handle's
 * pair laws and no tree (the theta -> 0 limit of Search_Tree_*,
 * tree.f90:721-1133).  targets: global indices (electrons 0..n_el-1, ions
 * n_el..n_el+n_ion-1).  Out (host): f (3*nt), epot (nt; 0.5*sum of V per
 * target).  Allocates its device scratch per call. */
int tree_gpu_direct(tree_gpu_handle* h, const int64_t* targets, int64_t nt,
                    double* f, double* epot);

/* Allocation-free direct sum.  No counterpart in the reference.  For callers
 * that cannot call cudaMalloc: a host program whose memory manager owns all
 * device memory and hands out only its own buffers, or code running where an
 * allocation would synchronise the device or is not permitted.  It computes
 * what tree_gpu_direct computes, but takes DEVICE pointers and no handle:
 *   d_x       positions, 3*(n_el+n_ion) doubles, electrons first (AoS xyz)
 *   d_targets nt global particle indices (int64)
 *   d_f, d_epot  outputs: 3*nt forces and nt values of 0.5*sum V
 *   stream    cudaStream_t to run on (NULL: the default stream)
 * Its scratch is a file-scope static device array of 8 MiB that every GPU
 * loading this library keeps until the process exits.  The array is committed
 * on a device when the library's direct-sum module is first loaded there:
 * with CUDA's default lazy module loading that is the first call of
 * tree_gpu_direct or tree_gpu_direct_static on that device (a caller whose
 * memory manager takes all free memory should make one such call, or set
 * CUDA_MODULE_LOADING=EAGER, before it does); later calls commit nothing.
 * nt may be at most TREE_GPU_DIRECT_STATIC_MAX_TARGETS (larger lists return
 * TREE_GPU_ERR_CAPACITY and do no work); an index outside [0, n) returns
 * TREE_GPU_ERR_ARG (it is replaced by 0 on the device, so nothing is read out
 * of bounds).  The first call on each device looks up the scratch address
 * (cudaGetSymbolAddress), so make that first call before any stream capture.
 * All calls share the one array and its contents persist between calls:
 * calls that overlap on the GPU (other streams or threads) race on it.  Each
 * launch's status is checked on its own, so an error left by the caller's
 * earlier work is neither reported nor cleared.  The call copies a 4-byte
 * error word to the host and synchronises `stream` before it returns. */
#define TREE_GPU_DIRECT_STATIC_MAX_TARGETS 65536
int tree_gpu_direct_static(const double* d_x, int64_t n_el, int64_t n_ion,
                           const tree_gpu_params* params,
                           const int64_t* d_targets, int64_t nt, double* d_f,
                           double* d_epot, void* stream);

/* Debug/parity: copies one species tree (0 electrons, 1 ions) of the last
 * build in pre-order (children 1..8, the reference's visiting order).
 * Per node: centre[3] (charge centre, or the particle for leaves), moments[10]
 * (qeff, D[3], Q[3], QQ[3]), rcrit (s/theta + dx; -1 for leaves), level,
 * skip (pre-order index past the subtree, tree-local), pt (particle index
 * for leaves, -1 for twigs).  Pass NULL buffers to query *n_nodes only. */
int tree_gpu_tree_dump(tree_gpu_handle* h, int32_t species, int64_t cap,
                       double* centre, double* moments, double* rcrit,
                       int32_t* level, int64_t* skip, int64_t* pt,
                       int64_t* n_nodes);

/* Debug: the combined tree of the mixed-precision path, rebuilt from the
 * current device positions with every record written (the step's own builds
 * write a twig's FP64 record only where the build reads it), in pre-order
 * (single-cloud handles of precision MIXED).  Per node:
 * centre[3] (the expansion centre: a twig's centroid, a leaf's particle),
 * moments[38] (a twig's FP64 record: n, Q, Dx, Dy, Dz, q_ion, Sxx, Syy, Szz,
 * Sxy, Syz, Szx with S = 1/2 sum q a a^T, T[10] in the order xxx yyy zzz xxy
 * xxz xyy yyz xzz yzz xyz, H[15] in the order xxxx yyyy zzzz xxxy xxxz xyyy
 * yyyz xzzz yzzz xxyy xxzz yyzz xxyz xyyz xyzz, 0; all zero for a leaf),
 * first and count (the node's range of sorted particles), level, parent
 * (-1 for the root);
 * sorted[4 * (n_el + n_ion)]: the sorted particles (x, y, z, 1 for an ion or
 * 0 for an electron).  NULL buffers are skipped; *n_nodes receives the node
 * count (pass all buffers NULL to query it). */
int tree_gpu_net_dump(tree_gpu_handle* h, int64_t cap, double* centre, double* moments,
                      int64_t* first, int64_t* count, int32_t* level, int64_t* parent,
                      double* sorted, int64_t* n_nodes);

/* Runs all later work of the handle on `stream` (a cudaStream_t; NULL
 * restores the handle's own stream).  No counterpart in the reference (its
 * work is on host threads); lets a caller order the force path with its own
 * device work and time it with events on the same stream. */
int tree_gpu_set_stream(tree_gpu_handle* h, void* stream);

/* Tunables of the mixed-precision walk: twigs holding at most `bucket`
 * particles (1..8) are summed particle by particle instead of being opened;
 * `blocks_per_sm` (1..4) sets the persistent grid of the walk without RDF
 * counts (the learned criterion's walk holds at most 2 blocks per SM and is
 * clamped there; with RDF counts the walk runs one block per SM); `order` (2..4) is the
 * far-field expansion order (quadrupole; octupole as well, the default 3; or
 * hexadecapole as well, 4).  A learned acceptance model predicts the error of
 * one order: load one trained at the order in use.
 * No counterpart in the reference; chosen by the autotuner (tree_b200/tune.py). */
int tree_gpu_set_tuning(tree_gpu_handle* h, int32_t bucket,
                        int32_t blocks_per_sm, int32_t order);

/* Local expansions of far cells in the mixed-precision walk.  An accepted
 * cell far from a target group (32 targets at most) is expanded once about
 * the group's centre to second order in the force (value, gradient, second
 * and third derivatives of its potential) instead of being evaluated at every
 * target; the group sums these expansions and each target evaluates the sum
 * once.  A cell is far when h/d <= max_ratio, h the group's half-diagonal and
 * d the distance from the group's centre to the cell's centroid; the added
 * force error is of order (h/d)^3 of that cell's field.  Default 0.08;
 * 0 evaluates every accepted cell at every target; at most 0.5.  No
 * counterpart in the reference, whose walks evaluate every accepted cell per
 * target (tree.f90:744-779). */
int tree_gpu_set_local_expansion(tree_gpu_handle* h, double max_ratio);

/* ---- learned multipole acceptance criterion (no counterpart in the
 * reference, whose criterion is the fixed s/theta + dx < r of tree.f90:743).
 * A 16 -> 64 -> 64 -> 1 network predicts log10 of the error of accepting a
 * cell for a target group, relative to the cell's gross monopole field.  A
 * cell that the fixed-theta test would open, with s/(d - dx) <= rho_hi, is
 * accepted anyway when the predicted error is at most eta * (smallest |F| of
 * the group at the previous step); features outside the training range keep
 * the fixed-theta decision.  Active when precision = MIXED and mac = LEARNED
 * and a model is loaded. */
#define TREE_GPU_MLP_PARAMS 5313 /* W1[16][64] b1[64] W2[64][64] b2[64] w3[64] b3 */
#define TREE_GPU_MLP_STATS 72    /* feature mean[16], 1/std[16], min[16], max[16],
                                    margins m_lo, m_hi (20% and 99.5% quantiles
                                    of label minus the pre-filter estimate),
                                    pre-filter coefficients c0..c4, 1 reserved */

/* Walks the combined tree of the current device positions with a fixed
 * theta drawn per target group from [theta_lo, theta_hi] and appends one
 * training sample (16 features, label, and (theta, rho)) per tested cell in
 * the band [rho_lo, rho_hi] holding at most max_count particles; the label
 * is the exact FP64 error of accepting it.  The sample buffer holds `cap`
 * samples (reallocated, and emptied, when cap changes); *n_total receives
 * the number held. */
int tree_gpu_mac_collect(tree_gpu_handle* h, double theta_lo, double theta_hi,
                         double rho_lo, double rho_hi, int32_t max_count,
                         float keep, uint64_t seed, int64_t cap,
                         int64_t* n_total);
/* Copies the collected samples out (NULL buffers: count only). */
int tree_gpu_mac_samples(tree_gpu_handle* h, float* feats, float* labels,
                         float* extra, int64_t cap, int64_t* n);
int tree_gpu_mac_clear(tree_gpu_handle* h);
/* Trains the network from scratch on the collected samples with the
 * BF16 tensor-core kernels (pinball loss at quantile tau, Adam, cosine decay)
 * and loads it; loss_per_epoch (epochs floats) may be NULL. */
int tree_gpu_mac_train(tree_gpu_handle* h, int32_t epochs, int32_t batch,
                       float lr, float tau, uint64_t seed,
                       float* loss_per_epoch);
int tree_gpu_mac_set_model(tree_gpu_handle* h, const float* params,
                           const float* stats);
int tree_gpu_mac_get_model(tree_gpu_handle* h, float* params, float* stats);
int tree_gpu_mac_config(tree_gpu_handle* h, float eta, float rho_lo,
                        float rho_hi);
/* Stand-alone network kernels (host buffers, device scratch per call), used to
 * check gradients and inference against a CPU implementation. */
int tree_gpu_mlp_grad(const float* X, const float* y, int64_t n,
                      const float* params, float tau, float* grad,
                      float* loss);
int tree_gpu_mlp_infer(const float* X, int64_t n, const float* params,
                       const float* stats, float* y);

int tree_gpu_timings(tree_gpu_handle* h, tree_gpu_timing* out);
const char* tree_gpu_last_error(tree_gpu_handle* h);
int tree_gpu_destroy(tree_gpu_handle* h);

/* Library build identifier (sm_100a + git describe at build time). */
const char* tree_gpu_version(void);

/* ---- ensembles of independent clouds (no counterpart in the reference,
 * which runs one cloud per job).  ncloud clouds (1..256) of uneven size share
 * one handle: one build (a forest, each cloud with its own root box), one
 * persistent walk launch and one integrator launch per step, replayed as a
 * CUDA graph.  Particles are cloud-major: cloud c holds n_el[c] electrons
 * then n_ion[c] ions; x, v, f are AoS double xyz over all particles.  Each
 * cloud keeps its own te, rs and RDF bin widths; theta, physics, mac and the
 * masses must agree across clouds; precision must be MIXED.  tree_gpu_step,
 * tree_gpu_run (without RDF), tree_gpu_set_tuning, tree_gpu_set_params
 * (theta and mac only), tree_gpu_mac_set_model / _config and
 * tree_gpu_timings work on ensemble handles; the species-split calls
 * (force, set/load/get_state, direct, tree_dump, mac_collect) return
 * TREE_GPU_ERR_ARG. */
int tree_gpu_ensemble_create(const tree_gpu_params* params, int32_t ncloud,
                             const int64_t* n_el, const int64_t* n_ion,
                             tree_gpu_handle** out);
/* Positions and velocities in, initial forces computed (Vinit). */
int tree_gpu_ensemble_set_state(tree_gpu_handle* h, const double* x,
                                const double* v);
/* Full state in (f NULL: forces computed as by set_state). */
int tree_gpu_ensemble_load_state(tree_gpu_handle* h, const double* x,
                                 const double* v, const double* f);
int tree_gpu_ensemble_get_state(tree_gpu_handle* h, double* x, double* v,
                                double* f);
/* Per-cloud (Epot_e, Epot_i, mv2_el, mv2_ion, rad_el, rad_ion) of the
 * current state, 6 x ncloud doubles (TEMPORAL per cloud). */
int tree_gpu_ensemble_sums(tree_gpu_handle* h, double* out);
/* FP64 direct sum inside one cloud; targets are cloud-local indices. */
int tree_gpu_ensemble_direct(tree_gpu_handle* h, int32_t cloud,
                             const int64_t* targets, int64_t nt, double* f,
                             double* epot);

#ifdef __cplusplus
}
#endif

#endif /* TREE_GPU_H */
