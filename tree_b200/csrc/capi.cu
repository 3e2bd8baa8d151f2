// capi.cu -- the extern "C" boundary (include/tree_gpu.h).
//
// Replaces SUBROUTINE Force (main.f90:506-701) and the VVerlet calls of the
// step loop (main.f90:125-131) for one GPU: one device-resident tree per
// species instead of the 8-rank octant decomposition and ghost-tree exchange.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/tree_gpu.h"
#include "build.h"
#include "direct.h"
#include "internal.cuh"
#include "kdk.h"
#include "mlp.h"
#include "walk.h"
#include "walk_mixed.h"

#ifndef TREE_GPU_VERSION_STR
#define TREE_GPU_VERSION_STR "tree_b200 sm_100a"
#endif

namespace {

constexpr double kHbar = 1.054571817e-34;  // J s
constexpr double kAmu = 1.66053906660e-27;  // kg
constexpr double kKbSi = 1.380649e-23;      // J/K
constexpr int kMaxClouds = 256;             // cloud id in at most 8 key bits

double kelbg_lambda_um(double mu_amu, double te) {
  return kHbar / std::sqrt(2.0 * mu_amu * kAmu * kKbSi * te) * 1e6;
}

struct EventSet {
  cudaEvent_t e[4];
};

// One captured step body (force + second kick [+ samples] [+ RDF fold]).
struct StepGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  EventSet ev{};
  bool has_ev = false;
  cudaGraphNode_t ev_node[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t epoch = 0;
  double dt = 0.0;
  int64_t launches = 0;  // kernels in one replay
  int64_t replays = 0;   // replays during the current call
};

}  // namespace

struct tree_gpu_handle {
  tree_gpu_params prm{};
  int64_t n_el = 0, n_ion = 0;
  int n = 0;
  int device = 0;
  cudaStream_t st = nullptr;      // stream all work is enqueued on
  cudaStream_t own_st = nullptr;  // the handle's own stream
  double* x = nullptr;
  double* v = nullptr;
  double* f = nullptr;
  double2* epot_part = nullptr;
  tg::BuildBuffers b{};
  tg::MixedBuffers mb{};
  tg::MixedTuning tune{};
  // learned MAC
  float* mlp_params = nullptr;   // kMlpParams FP32 master parameters
  float* mlp_stats = nullptr;    // mean[16] inv_std[16] fmin[16] fmax[16]
  tg::MlpPacked* mlp_packed = nullptr;
  bool has_model = false;
  bool has_fprev = false;        // h->f holds forces of the current positions' predecessor
  float mac_eta = 1e-5f, mac_rho_lo = 0.2f, mac_rho_hi = 0.9f;
  float* smp_feats = nullptr;    // collected training samples
  float* smp_labels = nullptr;
  float* smp_extra = nullptr;
  int32_t* smp_count = nullptr;
  int64_t smp_cap = 0;
  uint32_t* rdf = nullptr;
  unsigned long long* counters = nullptr;
  double* partial = nullptr;
  double* diag = nullptr;  // [0..3] epot, [4..7] kinetic sums
  int32_t* h_pinned = nullptr;  // small pinned readback area
  bool has_state = false;
  double lam[3] = {1, 1, 1};
  tree_gpu_timing timing{};
  std::vector<EventSet> events;
  std::string last_error;
  // step loop: CUDA graphs of the step body, [sample][last][rdf]
  StepGraph graphs[2][2][2];
  bool use_graphs = true;
  uint64_t epoch = 1;        // bumped whenever a captured argument may change
  bool capturing = false;    // a step body is being captured into a graph
  int64_t nloop = 0;         // ttime%Nloop: steps since the state was set
  double* series = nullptr;  // sample records of a run, 6 doubles each
  int32_t* series_count = nullptr;
  int series_cap = 0;
  unsigned long long* rdf64 = nullptr;  // RDF sums of a run (2 x kRdfBins)
  // ensemble of independent clouds (b.ens.nseg > 0)
  std::vector<tree_gpu_params> cloud_prm;
  std::vector<int64_t> cloud_ne, cloud_ni;
  int32_t* ens_start = nullptr;     // device, nseg + 1
  int32_t* ens_elec_end = nullptr;  // device, nseg
  int32_t* ens_roots = nullptr;     // device, nseg
  int32_t* ens_glvl = nullptr;      // device, nseg x kLevelSlots
  float4* cloud_pk = nullptr;       // device, 2 per cloud
  uint8_t* ion_flag = nullptr;      // device, per particle (ensembles)
  double* cloud_sums = nullptr;     // device, 6 per cloud
};

namespace {

int fail(tree_gpu_handle* h, int code, const std::string& msg) {
  if (h) h->last_error = msg;
  return code;
}

#define CK(call)                                                            \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return fail(h, TREE_GPU_ERR_CUDA,                                     \
                  std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

int check_params(const tree_gpu_params* p) {
  if (!p) return TREE_GPU_ERR_ARG;
  if (!(p->theta > 0.0) || !std::isfinite(p->theta)) return TREE_GPU_ERR_ARG;
  if (p->physics != TREE_GPU_PHYS_REF && p->physics != TREE_GPU_PHYS_KELBG)
    return TREE_GPU_ERR_ARG;
  if (p->precision != TREE_GPU_PREC_FP64 && p->precision != TREE_GPU_PREC_MIXED)
    return TREE_GPU_ERR_ARG;
  if (p->mac != TREE_GPU_MAC_FIXED && p->mac != TREE_GPU_MAC_LEARNED)
    return TREE_GPU_ERR_ARG;
  if (p->physics == TREE_GPU_PHYS_REF && !(p->rs > 0.0)) return TREE_GPU_ERR_ARG;
  if (p->physics == TREE_GPU_PHYS_KELBG &&
      (!(p->te > 0.0) || !(p->xm_el > 0.0) || !(p->xm_ion > 0.0)))
    return TREE_GPU_ERR_ARG;
  if (!(p->dx_ei > 0.0) || !(p->dx_ii > 0.0)) return TREE_GPU_ERR_ARG;
  return TREE_GPU_OK;
}

void set_lambdas(tree_gpu_handle* h) {
  const tree_gpu_params& p = h->prm;
  if (p.te > 0.0 && p.xm_el > 0.0 && p.xm_ion > 0.0) {
    h->lam[0] = kelbg_lambda_um(p.xm_el / 2.0, p.te);
    h->lam[1] = kelbg_lambda_um(p.xm_el * p.xm_ion / (p.xm_el + p.xm_ion), p.te);
    h->lam[2] = kelbg_lambda_um(p.xm_ion / 2.0, p.te);
  }
}

template <class T>
int dalloc(tree_gpu_handle* h, T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) count = 1;
  CK(cudaMalloc((void**)p, count * sizeof(T)));
  return 0;
}

int alloc_nodes(tree_gpu_handle* h, int cap) {
  tg::BuildBuffers& b = h->b;
  b.cap = cap;
  ++h->epoch;  // captured step graphs hold the old node pointers
  int rc = 0;
  if ((rc = dalloc(h, &b.node_c, cap))) return rc;
  if ((rc = dalloc(h, &b.node_m, 5 * (size_t)cap))) return rc;
  if ((rc = dalloc(h, &b.node_skip, cap))) return rc;
  if ((rc = dalloc(h, &b.node_pt, cap))) return rc;
  if ((rc = dalloc(h, &b.node_parent, cap))) return rc;
  if ((rc = dalloc(h, &b.node_nchild, cap))) return rc;
  if ((rc = dalloc(h, &b.node_done, cap))) return rc;
  if ((rc = dalloc(h, &b.node_level, cap))) return rc;
  if (tg::mixed_alloc_nodes(h->mb, cap))
    return fail(h, TREE_GPU_ERR_CUDA, "mixed node alloc");
  h->b.mx = tg::mixed_nodes(h->mb);
  return 0;
}

int alloc_all(tree_gpu_handle* h) {
  int n = h->n;
  tg::BuildBuffers& b = h->b;
  int rc = 0;
  if ((rc = dalloc(h, &h->x, 3 * (size_t)n))) return rc;
  if ((rc = dalloc(h, &h->v, 3 * (size_t)n))) return rc;
  if ((rc = dalloc(h, &h->f, 3 * (size_t)n))) return rc;
  if ((rc = dalloc(h, &h->epot_part, n))) return rc;
  if ((rc = dalloc(h, &b.keys, n))) return rc;
  if ((rc = dalloc(h, &b.keys_alt, n))) return rc;
  if ((rc = dalloc(h, &b.vals, n))) return rc;
  if ((rc = dalloc(h, &b.vals_alt, n))) return rc;
  if ((rc = dalloc(h, &b.L, n))) return rc;
  if ((rc = dalloc(h, &b.cnt, n))) return rc;
  if ((rc = dalloc(h, &b.off, (size_t)n + 1))) return rc;
  int rb = tg::radix_blocks(n);
  if ((rc = dalloc(h, &b.sort_hist, 256 * (size_t)rb))) return rc;
  int sp = tg::scan_partials_needed(256 * rb > n + 1 ? 256 * rb : n + 1);
  if ((rc = dalloc(h, &b.scan_partial, (size_t)sp + 1))) return rc;
  if ((rc = dalloc(h, &b.bbox, 12))) return rc;
  if ((rc = dalloc(h, &b.geom, 2))) return rc;
  if ((rc = dalloc(h, &b.bounds, 5))) return rc;
  if ((rc = dalloc(h, &b.err, 1))) return rc;
  if ((rc = dalloc(h, &h->rdf, 2 * (size_t)tg::kRdfBins))) return rc;
  if ((rc = dalloc(h, &h->counters, 16))) return rc;
  // [0..3] this step's walk counts, [4..7] running totals of the handle,
  // [8] this step's cells in local expansions, [9] their running total
  if (cudaMemset(h->counters, 0, 16 * sizeof(unsigned long long)) != cudaSuccess)
    return fail(h, TREE_GPU_ERR_CUDA, "counter initialisation failed");
  if ((rc = dalloc(h, &h->partial, 4 * (size_t)tg::kdk_partials_needed(n) + 4)))
    return rc;
  if ((rc = dalloc(h, &h->diag, 8))) return rc;
  CK(cudaMemsetAsync(h->diag, 0, 8 * sizeof(double), h->st));
  if (tg::mixed_alloc_particles(h->mb, n))
    return fail(h, TREE_GPU_ERR_CUDA, "mixed particle alloc");
  h->b.mx = tg::mixed_nodes(h->mb);
  int cap = 3 * n + 64;
  return alloc_nodes(h, cap);
}

void free_all(tree_gpu_handle* h) {
  tg::BuildBuffers& b = h->b;
  void* ptrs[] = {h->x, h->v, h->f, h->epot_part, b.keys, b.keys_alt, b.vals,
                  b.vals_alt, b.L, b.cnt, b.off, b.sort_hist, b.scan_partial,
                  b.bbox, b.geom, b.bounds, b.err, b.node_c, b.node_m,
                  b.node_skip, b.node_pt, b.node_parent, b.node_nchild,
                  b.node_done, b.node_level, h->rdf, h->counters, h->partial,
                  h->diag, h->mlp_params, h->mlp_stats, h->mlp_packed,
                  h->smp_feats, h->smp_labels, h->smp_extra, h->smp_count,
                  h->series, h->series_count, h->rdf64, h->ens_start,
                  h->ens_elec_end, h->ens_roots, h->ens_glvl, h->cloud_pk,
                  h->ion_flag, h->cloud_sums};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  tg::mixed_free(h->mb);
}

tg::TreeView tree_view(tree_gpu_handle* h) {
  tg::TreeView tv;
  tv.node_c = h->b.node_c;
  tv.node_m = h->b.node_m;
  tv.node_skip = h->b.node_skip;
  tv.node_pt = h->b.node_pt;
  tv.tree_bounds = h->b.bounds;
  return tv;
}

tg::WalkParams walk_params(tree_gpu_handle* h) {
  tg::WalkParams wp;
  wp.physics = h->prm.physics;
  wp.theta = h->prm.theta;
  wp.rs = h->prm.rs;
  wp.lam_ee = h->lam[0];
  wp.lam_ei = h->lam[1];
  wp.lam_ii = h->lam[2];
  wp.dx_ei = h->prm.dx_ei;
  wp.dx_ii = h->prm.dx_ii;
  return wp;
}

EventSet& events_for(tree_gpu_handle* h, size_t i) {
  while (h->events.size() <= i) {
    EventSet es;
    for (int k = 0; k < 4; ++k) cudaEventCreate(&es.e[k]);
    h->events.push_back(es);
  }
  return h->events[i];
}

// Records a timing event; inside a capture it becomes an event-record node
// of the graph, so every replay records it.
void record(tree_gpu_handle* h, cudaEvent_t e) {
  cudaEventRecordWithFlags(e, h->st, h->capturing ? cudaEventRecordExternal
                                                  : cudaEventRecordDefault);
}

// Enqueues build + walk + potential-energy sum on the handle's stream.
void enqueue_force(tree_gpu_handle* h, bool with_rdf, EventSet* ev) {
  cudaStream_t st = h->st;
  if (ev) record(h, ev->e[0]);
  const int mode = h->prm.precision == TREE_GPU_PREC_FP64 ? 0 : 1;
  h->timing.launches +=
      tg::build_trees(h->b, h->x, h->n, (int)h->n_el, h->prm.theta, mode, st);
  if (ev) record(h, ev->e[1]);
  cudaMemsetAsync(h->counters, 0, 4 * sizeof(unsigned long long), st);
  cudaMemsetAsync(h->counters + 8, 0, sizeof(unsigned long long), st);
  if (with_rdf)
    cudaMemsetAsync(h->rdf, 0, 2 * sizeof(uint32_t) * tg::kRdfBins, st);
  tg::TreeView tv = tree_view(h);
  tg::WalkParams wp = walk_params(h);
  if (h->prm.precision == TREE_GPU_PREC_FP64) {
    tg::walk64(h->x, h->n, (int)h->n_el, h->b.vals, tv, wp, h->f,
               h->epot_part, with_rdf ? h->rdf : nullptr, h->counters,
               h->b.err, st);
    h->timing.launches += h->n > 0 ? 1 : 0;
  } else {
    tg::LearnedMac lm;
    const bool use_learned = h->prm.mac == TREE_GPU_MAC_LEARNED && h->has_model &&
                             h->has_fprev;
    if (use_learned) {
      lm.packed = h->mlp_packed;
      lm.fmin = h->mlp_stats + 32;
      lm.fmax = h->mlp_stats + 48;
      lm.margins = h->mlp_stats + 64;
      lm.f_prev = h->f;  // each target's previous force, read before it is overwritten
      lm.eta = h->mac_eta;
      lm.rho_lo = h->mac_rho_lo;
      lm.rho_hi = h->mac_rho_hi;
    }
    // the walk, and with the learned criterion its per-cell pre-filter pass
    h->timing.launches +=
        tg::walk_mixed(h->mb, h->b, h->x, h->n, (int)h->n_el, tv, wp, h->tune,
                       use_learned ? &lm : nullptr, h->b.ens, h->cloud_pk, h->f, h->epot_part,
                       with_rdf ? h->rdf : nullptr, h->counters, h->b.err, st);
  }
  if (ev) record(h, ev->e[2]);
  h->timing.launches += 2;  // epot partial/sum
  tg::epot_sum(h->epot_part, h->n, h->partial, h->diag, h->counters, st);
}

// Reads the error word and node counts after a synchronised call.
int check_device_status(tree_gpu_handle* h, bool* grow) {
  *grow = false;
  int32_t* hp = h->h_pinned;
  CK(cudaMemcpyAsync(hp, h->b.err, sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(hp + 1, h->b.bounds, 4 * sizeof(int32_t),
                     cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  int32_t err = hp[0];
  h->timing.n_nodes = hp[1 + 3];
  if (err & tg::kErrNonFinite)
    return fail(h, TREE_GPU_ERR_NONFINITE, "non-finite particle position");
  if (err & tg::kErrDepth)
    return fail(h, TREE_GPU_ERR_DEPTH,
                "two same-species particles share a 42-level cell");
  if (err & tg::kErrCapacity) {
    *grow = true;
    return TREE_GPU_OK;
  }
  if (err & tg::kErrWalk) return fail(h, TREE_GPU_ERR_WALK, "walk guard tripped");
  return TREE_GPU_OK;
}

int grow_nodes(tree_gpu_handle* h) {
  int need = h->h_pinned[1 + 3];
  if (need <= h->b.cap) need = h->b.cap;
  int64_t cap = (int64_t)need + need / 4 + 64;
  if (cap > 0x7fffffff) return fail(h, TREE_GPU_ERR_CAPACITY, "node count overflow");
  CK(cudaStreamSynchronize(h->st));
  return alloc_nodes(h, (int)cap);
}

void read_counters(tree_gpu_handle* h) {
  unsigned long long c[16] = {};
  cudaMemcpy(c, h->counters, sizeof(c), cudaMemcpyDeviceToHost);
  h->timing.n_m2p = (int64_t)c[0];
  h->timing.n_p2p = (int64_t)c[1];
  h->timing.n_mac_net = (int64_t)c[2];
  h->timing.n_mac_fallback = (int64_t)c[3];
  h->timing.n_m2p_total = (int64_t)c[4];
  h->timing.n_p2p_total = (int64_t)c[5];
  h->timing.n_mac_net_total = (int64_t)c[6];
  h->timing.n_local = (int64_t)c[8];
  h->timing.n_local_total = (int64_t)c[9];
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();  // not recorded: no time, and no error left behind
    ms = 0.f;
  }
  return ms;
}

// Computes forces of the current device positions, growing the node arrays
// when the tree did not fit.
int force_device(tree_gpu_handle* h, bool with_rdf) {
  for (int attempt = 0; attempt < 3; ++attempt) {
    EventSet& ev = events_for(h, 0);
    enqueue_force(h, with_rdf, &ev);
    CK(cudaGetLastError());
    bool grow = false;
    int rc = check_device_status(h, &grow);
    if (rc) return rc;
    if (!grow) {
      h->timing.ms_build += elapsed(ev.e[0], ev.e[1]);
      h->timing.ms_walk += elapsed(ev.e[1], ev.e[2]);
      h->timing.ms_total += elapsed(ev.e[0], ev.e[2]);
      h->timing.calls += 1;
      read_counters(h);
      return TREE_GPU_OK;
    }
    if ((rc = grow_nodes(h))) return rc;
  }
  return fail(h, TREE_GPU_ERR_CAPACITY, "node capacity growth did not converge");
}

// One step of the main loop after the first half kick: Force, the second
// half kick fused with the next first half kick and drift (unless last), the
// kinetic sums and a sample record on sample steps, the RDF fold.
void enqueue_step_body(tree_gpu_handle* h, double dt, bool sample, bool last,
                       bool rdf, EventSet* ev) {
  const tree_gpu_params& p = h->prm;
  const int n = h->n, ne = (int)h->n_el;
  enqueue_force(h, rdf, ev);
  tg::kick2(h->x, h->v, h->f, n, ne, h->ion_flag, dt, p.xm_el, p.xm_ion, sample,
            !last, h->partial, h->diag + 4, h->st);
  h->timing.launches += n > 0 ? (sample ? 2 : 1) : 0;
  if (rdf) {
    tg::rdf_fold(h->rdf, h->rdf64, h->st);
    h->timing.launches += 1;
  }
  if (sample && h->series) {
    tg::sample_append(h->diag, h->series, h->series_count, h->series_cap, h->st);
    h->timing.launches += 1;
  }
  if (ev) record(h, ev->e[3]);
}

// The captured graph of a step-body variant, captured on first use or after
// any argument it holds changed; nullptr when capture is not possible on
// this stream (the caller then enqueues the body directly).
StepGraph* graph_for(tree_gpu_handle* h, double dt, bool sample, bool last, bool rdf) {
  StepGraph& g = h->graphs[sample][last][rdf];
  if (g.exec && g.epoch == h->epoch && g.dt == dt) return &g;
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
  if (!g.has_ev) {
    for (int k = 0; k < 4; ++k) cudaEventCreate(&g.ev.e[k]);
    g.has_ev = true;
  }
  if (cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const int64_t l0 = h->timing.launches;
  h->capturing = true;
  enqueue_step_body(h, dt, sample, last, rdf, &g.ev);
  h->capturing = false;
  g.launches = h->timing.launches - l0;
  h->timing.launches = l0;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->st, &graph);
  if (e != cudaSuccess || graph == nullptr) {
    cudaGetLastError();
    if (graph) cudaGraphDestroy(graph);
    return nullptr;
  }
  // the event-record nodes, so each replay can record into its own events
  size_t nn = 0;
  cudaGraphGetNodes(graph, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) cudaGraphGetNodes(graph, nodes.data(), &nn);
  for (int k = 0; k < 4; ++k) g.ev_node[k] = nullptr;
  for (cudaGraphNode_t nd : nodes) {
    cudaGraphNodeType ty;
    cudaEvent_t evn = nullptr;
    if (cudaGraphNodeGetType(nd, &ty) != cudaSuccess || ty != cudaGraphNodeTypeEventRecord)
      continue;
    if (cudaGraphEventRecordNodeGetEvent(nd, &evn) != cudaSuccess) continue;
    for (int k = 0; k < 4; ++k)
      if (evn == g.ev.e[k]) g.ev_node[k] = nd;
  }
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(graph);
    g.exec = nullptr;
    return nullptr;
  }
  g.graph = graph;
  g.epoch = h->epoch;
  g.dt = dt;
  return &g;
}

void free_graphs(tree_gpu_handle* h) {
  for (auto& a : h->graphs)
    for (auto& b2 : a)
      for (StepGraph& g : b2) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        if (g.has_ev)
          for (int k = 0; k < 4; ++k) cudaEventDestroy(g.ev.e[k]);
        g = StepGraph();
      }
}

// The step loop of main.f90:123-160 for nsteps steps.  Step Nloop samples
// when nsamp > 0 and Nloop % nsamp == 0 (vverlet.f90:81, main.f90:150), and
// always on the last step when sample_last; samples go to the series buffer
// when it is set.  With rdf, the near-field pair counts of every step are
// added to h->rdf64.
int run_impl(tree_gpu_handle* h, double dt, int32_t nsteps, int32_t nsamp,
             bool sample_last, bool rdf) {
  const int n = h->n, ne = (int)h->n_el;
  const tree_gpu_params& p = h->prm;
  events_for(h, (size_t)nsteps + 1);  // grow first: references below stay valid
  EventSet& et = events_for(h, 0);
  for (auto& a : h->graphs)
    for (auto& b2 : a)
      for (StepGraph& g : b2) g.replays = 0;
  std::vector<char> own_ev((size_t)nsteps, 0);  // step s recorded events[1 + s]
  cudaEventRecord(et.e[0], h->st);
  tg::kick_drift(h->x, h->v, h->f, n, ne, h->ion_flag, dt, p.xm_el, p.xm_ion, h->st);
  h->timing.launches += n > 0 ? 1 : 0;
  for (int s = 0; s < nsteps; ++s) {
    const int64_t nl = h->nloop + s + 1;
    const bool last = s == nsteps - 1;
    const bool sample = (nsamp > 0 && nl % nsamp == 0) || (sample_last && last);
    StepGraph* g = h->use_graphs ? graph_for(h, dt, sample, last, rdf) : nullptr;
    EventSet& ev = events_for(h, 1 + (size_t)s);
    if (g) {
      // point the replay's event-record nodes at this step's events
      bool own = true;
      for (int k = 0; k < 4; ++k)
        own = own && g->ev_node[k] &&
              cudaGraphExecEventRecordNodeSetEvent(g->exec, g->ev_node[k], ev.e[k]) ==
                  cudaSuccess;
      if (!own) cudaGetLastError();
      own_ev[s] = own ? 1 : 0;
      CK(cudaGraphLaunch(g->exec, h->st));
      g->replays += own ? 0 : 1;
      h->timing.launches += g->launches;
    } else {
      own_ev[s] = 1;
      enqueue_step_body(h, dt, sample, last, rdf, &ev);
    }
  }
  cudaEventRecord(et.e[1], h->st);
  CK(cudaGetLastError());
  bool grow = false;
  int rc = check_device_status(h, &grow);
  if (rc) return rc;
  if (grow) {
    // The positions already moved; a capacity miss means the forces of this
    // batch are invalid.  Report it: the caller restores state and retries.
    if ((rc = grow_nodes(h))) return rc;
    return fail(h, TREE_GPU_ERR_CAPACITY,
                "node capacity grew during step; state must be reloaded");
  }
  // phase times from each step's own events; a replay whose event nodes could
  // not be retargeted counts with its variant's last replay
  for (int s = 0; s < nsteps; ++s) {
    if (!own_ev[s]) continue;
    EventSet& ev = events_for(h, 1 + (size_t)s);
    h->timing.ms_build += elapsed(ev.e[0], ev.e[1]);
    h->timing.ms_walk += elapsed(ev.e[1], ev.e[2]);
  }
  for (auto& a : h->graphs)
    for (auto& b2 : a)
      for (StepGraph& g : b2)
        if (g.replays > 0) {
          h->timing.ms_build += g.replays * elapsed(g.ev.e[0], g.ev.e[1]);
          h->timing.ms_walk += g.replays * elapsed(g.ev.e[1], g.ev.e[2]);
        }
  h->timing.ms_total += elapsed(et.e[0], et.e[1]);
  h->timing.calls += nsteps;
  h->nloop += nsteps;
  read_counters(h);
  return TREE_GPU_OK;
}

}  // namespace

extern "C" {

int tree_gpu_create(const tree_gpu_params* params, int64_t n_el, int64_t n_ion,
                    tree_gpu_handle** out) {
  if (!out) return TREE_GPU_ERR_ARG;
  *out = nullptr;
  if (check_params(params) != TREE_GPU_OK) return TREE_GPU_ERR_ARG;
  if (n_el < 0 || n_ion < 0 || n_el + n_ion > (int64_t)0x7fffffff / 4)
    return TREE_GPU_ERR_ARG;
  tree_gpu_handle* h = new (std::nothrow) tree_gpu_handle();
  if (!h) return TREE_GPU_ERR_ARG;
  h->prm = *params;
  h->n_el = n_el;
  h->n_ion = n_ion;
  h->n = (int)(n_el + n_ion);
  set_lambdas(h);
  int rc = TREE_GPU_OK;
  do {
    if (cudaGetDevice(&h->device) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "no CUDA device");
      break;
    }
    if (cudaStreamCreateWithFlags(&h->own_st, cudaStreamNonBlocking) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "stream create failed");
      break;
    }
    h->st = h->own_st;
    if (cudaMallocHost((void**)&h->h_pinned, 64) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "pinned alloc failed");
      break;
    }
    rc = alloc_all(h);
  } while (0);
  if (rc != TREE_GPU_OK) {
    tree_gpu_destroy(h);
    return rc;
  }
  *out = h;
  return TREE_GPU_OK;
}

int tree_gpu_set_params(tree_gpu_handle* h, const tree_gpu_params* params) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (check_params(params) != TREE_GPU_OK)
    return fail(h, TREE_GPU_ERR_ARG, "invalid parameters");
  if (h->b.ens.nseg > 0) {
    // an ensemble keeps its clouds' physics; theta and the criterion change
    if (params->precision != TREE_GPU_PREC_MIXED)
      return fail(h, TREE_GPU_ERR_ARG, "ensembles run the mixed path only");
    h->prm.theta = params->theta;
    h->prm.mac = params->mac;
    for (tree_gpu_params& c : h->cloud_prm) {
      c.theta = params->theta;
      c.mac = params->mac;
    }
    ++h->epoch;
    return TREE_GPU_OK;
  }
  h->prm = *params;
  set_lambdas(h);
  ++h->epoch;
  return TREE_GPU_OK;
}

int tree_gpu_force(tree_gpu_handle* h, const double* x_el, const double* x_ion,
                   double* f_el, double* f_ion, double* epot_e, double* epot_i,
                   int64_t* rdf_ei, int64_t* rdf_ii) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  if ((h->n_el && (!x_el || !f_el)) || (h->n_ion && (!x_ion || !f_ion)))
    return fail(h, TREE_GPU_ERR_ARG, "null particle buffer");
  const size_t be = 3 * sizeof(double) * (size_t)h->n_el;
  const size_t bi = 3 * sizeof(double) * (size_t)h->n_ion;
  if (be) CK(cudaMemcpyAsync(h->x, x_el, be, cudaMemcpyHostToDevice, h->st));
  if (bi)
    CK(cudaMemcpyAsync(h->x + 3 * h->n_el, x_ion, bi, cudaMemcpyHostToDevice, h->st));
  bool with_rdf = rdf_ei || rdf_ii;
  int rc;
  if (h->prm.mac == TREE_GPU_MAC_LEARNED && h->prm.precision == TREE_GPU_PREC_MIXED) {
    // new positions: a fixed-theta pass gives the force magnitudes the learned
    // criterion budgets against, then the learned pass
    h->has_fprev = false;
    if ((rc = force_device(h, false))) return rc;
    h->has_fprev = true;
  }
  rc = force_device(h, with_rdf);
  h->has_fprev = false;
  h->has_state = false;  // the device positions are now this call's, not a state
  if (rc) return rc;
  if (be) CK(cudaMemcpyAsync(f_el, h->f, be, cudaMemcpyDeviceToHost, h->st));
  if (bi)
    CK(cudaMemcpyAsync(f_ion, h->f + 3 * h->n_el, bi, cudaMemcpyDeviceToHost, h->st));
  double ep[4];
  CK(cudaMemcpyAsync(ep, h->diag, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  std::vector<uint32_t> hr;
  if (with_rdf) {
    hr.resize(2 * (size_t)tg::kRdfBins);
    CK(cudaMemcpyAsync(hr.data(), h->rdf, hr.size() * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  if (epot_e) *epot_e = ep[0];
  if (epot_i) *epot_i = ep[1];
  if (with_rdf) {
    for (int i = 0; i < tg::kRdfBins; ++i) {
      if (rdf_ei) rdf_ei[i] += hr[i];
      if (rdf_ii) rdf_ii[i] += hr[tg::kRdfBins + i];
    }
  }
  return TREE_GPU_OK;
}

int tree_gpu_set_state(tree_gpu_handle* h, const double* x_el,
                       const double* v_el, const double* x_ion,
                       const double* v_ion) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  if ((h->n_el && (!x_el || !v_el)) || (h->n_ion && (!x_ion || !v_ion)))
    return fail(h, TREE_GPU_ERR_ARG, "null particle buffer");
  const size_t be = 3 * sizeof(double) * (size_t)h->n_el;
  const size_t bi = 3 * sizeof(double) * (size_t)h->n_ion;
  if (be) {
    CK(cudaMemcpyAsync(h->x, x_el, be, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->v, v_el, be, cudaMemcpyHostToDevice, h->st));
  }
  if (bi) {
    CK(cudaMemcpyAsync(h->x + 3 * h->n_el, x_ion, bi, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->v + 3 * h->n_el, v_ion, bi, cudaMemcpyHostToDevice, h->st));
  }
  h->has_fprev = false;  // initial forces with the fixed-theta test
  int rc = force_device(h, false);
  if (rc) return rc;
  h->has_state = true;
  h->has_fprev = true;
  h->nloop = 0;
  return TREE_GPU_OK;
}

int tree_gpu_load_state(tree_gpu_handle* h, const double* x_el,
                        const double* v_el, const double* f_el,
                        const double* x_ion, const double* v_ion,
                        const double* f_ion) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  if ((h->n_el && (!x_el || !v_el || !f_el)) ||
      (h->n_ion && (!x_ion || !v_ion || !f_ion)))
    return fail(h, TREE_GPU_ERR_ARG, "null particle buffer");
  const size_t be = 3 * sizeof(double) * (size_t)h->n_el;
  const size_t bi = 3 * sizeof(double) * (size_t)h->n_ion;
  const size_t oi = 3 * (size_t)h->n_el;
  if (be) {
    CK(cudaMemcpyAsync(h->x, x_el, be, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->v, v_el, be, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->f, f_el, be, cudaMemcpyHostToDevice, h->st));
  }
  if (bi) {
    CK(cudaMemcpyAsync(h->x + oi, x_ion, bi, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->v + oi, v_ion, bi, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->f + oi, f_ion, bi, cudaMemcpyHostToDevice, h->st));
  }
  h->has_state = true;
  h->has_fprev = true;
  h->nloop = 0;
  return TREE_GPU_OK;
}

int tree_gpu_step(tree_gpu_handle* h, double dt, int32_t nsteps,
                  tree_gpu_diag* out) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (!h->has_state) return fail(h, TREE_GPU_ERR_STATE, "tree_gpu_set_state first");
  if (nsteps < 0 || !std::isfinite(dt)) return fail(h, TREE_GPU_ERR_ARG, "bad dt/nsteps");
  if (nsteps == 0) return TREE_GPU_OK;
  double* keep = h->series;
  h->series = nullptr;  // no sample records, only the last step's sums
  int rc = run_impl(h, dt, nsteps, 0, true, false);
  h->series = keep;
  if (rc) return rc;
  if (out) {
    double d[8];
    CK(cudaMemcpy(d, h->diag, sizeof(d), cudaMemcpyDeviceToHost));
    out->epot_e = d[0];
    out->epot_i = d[1];
    out->mv2_el = d[4];
    out->rad_el = d[5];
    out->mv2_ion = d[6];
    out->rad_ion = d[7];
    out->steps_done = nsteps;
  }
  return TREE_GPU_OK;
}

int tree_gpu_run(tree_gpu_handle* h, double dt, int32_t nsteps, int32_t nsamp,
                 tree_gpu_sample* series, int32_t series_cap, int32_t* n_series,
                 int64_t* rdf_ei, int64_t* rdf_ii) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (!h->has_state) return fail(h, TREE_GPU_ERR_STATE, "tree_gpu_set_state first");
  if (nsteps < 0 || nsamp < 0 || series_cap < 0 || !std::isfinite(dt))
    return fail(h, TREE_GPU_ERR_ARG, "bad dt/nsteps/nsamp");
  if (n_series) *n_series = 0;
  if (nsteps == 0) return TREE_GPU_OK;
  const bool rdf = rdf_ei || rdf_ii;
  if (rdf && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "RDF counts are per cloud: not kept for ensembles");
  // sample steps of this call, and room for their records
  int64_t nsamples = 0;
  if (nsamp > 0) nsamples = (h->nloop + nsteps) / nsamp - h->nloop / nsamp;
  const bool want_series = series && series_cap > 0 && nsamples > 0;
  if (want_series && nsamples > h->series_cap) {
    const int cap = (int)std::min<int64_t>(nsamples + 16, 1 << 24);
    if (dalloc(h, &h->series, 6 * (size_t)cap)) return TREE_GPU_ERR_CUDA;
    if (!h->series_count && dalloc(h, &h->series_count, 1)) return TREE_GPU_ERR_CUDA;
    h->series_cap = cap;
    ++h->epoch;
  }
  if (rdf && !h->rdf64) {
    if (dalloc(h, &h->rdf64, 2 * (size_t)tg::kRdfBins)) return TREE_GPU_ERR_CUDA;
    ++h->epoch;
  }
  if (rdf) CK(cudaMemsetAsync(h->rdf64, 0, 2 * sizeof(unsigned long long) * tg::kRdfBins, h->st));
  if (h->series_count) CK(cudaMemsetAsync(h->series_count, 0, sizeof(int32_t), h->st));
  double* keep = h->series;
  if (!want_series) h->series = nullptr;  // sample steps still refresh the sums
  const int64_t nloop0 = h->nloop;
  int rc = run_impl(h, dt, nsteps, nsamp, false, rdf);
  h->series = keep;
  if (rc) return rc;
  if (want_series) {
    int32_t cnt = 0;
    CK(cudaMemcpy(&cnt, h->series_count, sizeof(int32_t), cudaMemcpyDeviceToHost));
    const int32_t m = std::min<int32_t>(cnt, series_cap);
    std::vector<double> buf(6 * (size_t)std::max<int32_t>(m, 1));
    if (m) CK(cudaMemcpy(buf.data(), h->series, 6 * sizeof(double) * m, cudaMemcpyDeviceToHost));
    int64_t nl = (nloop0 / nsamp + 1) * nsamp;  // first sample step of the call
    for (int32_t k = 0; k < m; ++k, nl += nsamp) {
      series[k].nloop = nl;
      series[k].epot_e = buf[6 * k];
      series[k].epot_i = buf[6 * k + 1];
      series[k].mv2_el = buf[6 * k + 2];
      series[k].mv2_ion = buf[6 * k + 3];
      series[k].rad_el = buf[6 * k + 4];
      series[k].rad_ion = buf[6 * k + 5];
    }
    if (n_series) *n_series = m;
  }
  if (rdf) {
    std::vector<unsigned long long> hr(2 * (size_t)tg::kRdfBins);
    CK(cudaMemcpy(hr.data(), h->rdf64, hr.size() * sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost));
    for (int i = 0; i < tg::kRdfBins; ++i) {
      if (rdf_ei) rdf_ei[i] += (int64_t)hr[i];
      if (rdf_ii) rdf_ii[i] += (int64_t)hr[tg::kRdfBins + i];
    }
  }
  return TREE_GPU_OK;
}

int tree_gpu_set_graphs(tree_gpu_handle* h, int32_t enable) {
  if (!h) return TREE_GPU_ERR_ARG;
  h->use_graphs = enable != 0;
  return TREE_GPU_OK;
}

int tree_gpu_get_nloop(tree_gpu_handle* h, int64_t* nloop) {
  if (!h || !nloop) return TREE_GPU_ERR_ARG;
  *nloop = h->nloop;
  return TREE_GPU_OK;
}

int tree_gpu_get_state(tree_gpu_handle* h, double* x_el, double* v_el,
                       double* f_el, double* x_ion, double* v_ion,
                       double* f_ion) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  const size_t be = 3 * sizeof(double) * (size_t)h->n_el;
  const size_t bi = 3 * sizeof(double) * (size_t)h->n_ion;
  const size_t oi = 3 * (size_t)h->n_el;
  if (be) {
    if (x_el) CK(cudaMemcpyAsync(x_el, h->x, be, cudaMemcpyDeviceToHost, h->st));
    if (v_el) CK(cudaMemcpyAsync(v_el, h->v, be, cudaMemcpyDeviceToHost, h->st));
    if (f_el) CK(cudaMemcpyAsync(f_el, h->f, be, cudaMemcpyDeviceToHost, h->st));
  }
  if (bi) {
    if (x_ion) CK(cudaMemcpyAsync(x_ion, h->x + oi, bi, cudaMemcpyDeviceToHost, h->st));
    if (v_ion) CK(cudaMemcpyAsync(v_ion, h->v + oi, bi, cudaMemcpyDeviceToHost, h->st));
    if (f_ion) CK(cudaMemcpyAsync(f_ion, h->f + oi, bi, cudaMemcpyDeviceToHost, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return TREE_GPU_OK;
}

int tree_gpu_direct(tree_gpu_handle* h, const int64_t* targets, int64_t nt,
                    double* f, double* epot) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  if (nt < 0 || nt > 0x7fffffff || (nt && (!targets || !f || !epot)))
    return fail(h, TREE_GPU_ERR_ARG, "bad target list");
  if (nt == 0) return TREE_GPU_OK;
  for (int64_t i = 0; i < nt; ++i)
    if (targets[i] < 0 || targets[i] >= h->n)
      return fail(h, TREE_GPU_ERR_ARG, "target index out of range");
  int nch = tg::direct_chunks(h->n, (int)nt);
  int64_t* d_t = nullptr;
  double4* d_part = nullptr;
  double* d_f = nullptr;
  double* d_e = nullptr;
  int rc = TREE_GPU_OK;
  do {
    if (cudaMalloc(&d_t, nt * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&d_part, (size_t)nch * nt * sizeof(double4)) != cudaSuccess ||
        cudaMalloc(&d_f, 3 * nt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_e, nt * sizeof(double)) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "direct-sum scratch allocation failed");
      break;
    }
    cudaMemcpyAsync(d_t, targets, nt * sizeof(int64_t), cudaMemcpyHostToDevice, h->st);
    h->timing.launches += tg::direct_sum(h->x, h->n, (int)h->n_el, d_t, (int)nt,
                                         walk_params(h), nch, d_part, d_f, d_e,
                                         h->st);
    cudaMemcpyAsync(f, d_f, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    cudaMemcpyAsync(epot, d_e, nt * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) rc = fail(h, TREE_GPU_ERR_CUDA, cudaGetErrorString(e));
  } while (0);
  cudaFree(d_t);
  cudaFree(d_part);
  cudaFree(d_f);
  cudaFree(d_e);
  return rc;
}

int tree_gpu_tree_dump(tree_gpu_handle* h, int32_t species, int64_t cap,
                       double* centre, double* moments, double* rcrit,
                       int32_t* level, int64_t* skip, int64_t* pt,
                       int64_t* n_nodes) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h || (species != 0 && species != 1)) return TREE_GPU_ERR_ARG;
  int32_t bnd[4];
  CK(cudaMemcpy(bnd, h->b.bounds, sizeof(bnd), cudaMemcpyDeviceToHost));
  int lo = bnd[species], hi = bnd[species + 1];
  int m = hi - lo;
  if (n_nodes) *n_nodes = m;
  if (!centre && !moments && !rcrit && !level && !skip && !pt) return TREE_GPU_OK;
  if (cap < m) return fail(h, TREE_GPU_ERR_ARG, "dump buffer too small");
  std::vector<double4> c(m);
  std::vector<double2> mm(5 * (size_t)m);
  std::vector<int32_t> sk(m), p(m);
  std::vector<int8_t> lv(m);
  if (m) {
    CK(cudaMemcpy(c.data(), h->b.node_c + lo, m * sizeof(double4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(mm.data(), h->b.node_m + 5 * (size_t)lo, 5 * m * sizeof(double2),
                  cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sk.data(), h->b.node_skip + lo, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(p.data(), h->b.node_pt + lo, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(lv.data(), h->b.node_level + lo, m * sizeof(int8_t), cudaMemcpyDeviceToHost));
  }
  for (int i = 0; i < m; ++i) {
    if (centre) {
      centre[3 * i] = c[i].x;
      centre[3 * i + 1] = c[i].y;
      centre[3 * i + 2] = c[i].z;
    }
    if (rcrit) rcrit[i] = c[i].w;
    if (moments)
      for (int j = 0; j < 5; ++j) {
        moments[10 * i + 2 * j] = mm[5 * (size_t)i + j].x;
        moments[10 * i + 2 * j + 1] = mm[5 * (size_t)i + j].y;
      }
    if (level) level[i] = lv[i];
    if (skip) skip[i] = (int64_t)sk[i] - lo;
    if (pt) {
      int64_t q = p[i];
      if (q >= 0 && species == 1) q -= h->n_el;  // species-local index
      pt[i] = q;
    }
  }
  return TREE_GPU_OK;
}

// The combined tree of the current device positions with every twig's FP64
// record written (the sampler's labels and the dump read them).
static int build_full_records(tree_gpu_handle* h) {
  for (int attempt = 0; attempt < 3; ++attempt) {
    h->timing.launches += tg::build_trees(h->b, h->x, h->n, (int)h->n_el,
                                          h->prm.theta, 1, h->st, true);
    bool grow = false;
    int rc = check_device_status(h, &grow);
    if (rc) return rc;
    if (!grow) break;
    if ((rc = grow_nodes(h))) return rc;
    if (attempt == 2) return fail(h, TREE_GPU_ERR_CAPACITY, "capacity");
  }
  return TREE_GPU_OK;
}

int tree_gpu_net_dump(tree_gpu_handle* h, int64_t cap, double* centre, double* moments,
                      int64_t* first, int64_t* count, int32_t* level, int64_t* parent,
                      double* sorted, int64_t* n_nodes) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: no combined-tree dump");
  if (h->prm.precision != TREE_GPU_PREC_MIXED)
    return fail(h, TREE_GPU_ERR_ARG, "the combined tree exists on the mixed path only");
  if (h->n == 0) return fail(h, TREE_GPU_ERR_STATE, "no particles");
  if (int rc = build_full_records(h)) return rc;
  int32_t bnd[4];
  CK(cudaMemcpy(bnd, h->b.bounds, sizeof(bnd), cudaMemcpyDeviceToHost));
  const int m = std::min(bnd[2], h->b.cap);
  if (n_nodes) *n_nodes = m;
  if (!centre && !moments && !first && !count && !level && !parent && !sorted)
    return TREE_GPU_OK;
  if (cap < m) return fail(h, TREE_GPU_ERR_ARG, "dump buffer too small");
  std::vector<double4> c(m);
  std::vector<double2> mm((size_t)tg::kM64 * m);
  std::vector<int32_t> fi(m), co(m), pt(m), pa(m);
  std::vector<int8_t> lv(m);
  if (m) {
    CK(cudaMemcpy(c.data(), h->b.node_c, m * sizeof(double4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(mm.data(), h->b.mx.m64, (size_t)tg::kM64 * m * sizeof(double2),
                  cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(fi.data(), h->b.mx.first, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(co.data(), h->b.mx.count, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pt.data(), h->b.node_pt, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pa.data(), h->b.node_parent, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(lv.data(), h->b.node_level, m * sizeof(int8_t), cudaMemcpyDeviceToHost));
  }
  for (int i = 0; i < m; ++i) {
    if (parent) parent[i] = pa[i];
    if (centre) {
      centre[3 * (size_t)i] = c[i].x;
      centre[3 * (size_t)i + 1] = c[i].y;
      centre[3 * (size_t)i + 2] = c[i].z;
    }
    if (moments) {
      // the FP64 record (n, Q) (Dx, Dy) (Dz, q_ion) (Sxx, Syy) (Szz, Sxy) (Syz, Szx) T H
      double* o = moments + 38 * (size_t)i;
      const bool leaf = pt[i] >= 0;
      for (int u = 0; u < tg::kM64; ++u) {
        o[2 * u] = leaf ? 0.0 : mm[(size_t)tg::kM64 * i + u].x;
        o[2 * u + 1] = leaf ? 0.0 : mm[(size_t)tg::kM64 * i + u].y;
      }
    }
    if (first) first[i] = fi[i];
    if (count) count[i] = co[i];
    if (level) level[i] = lv[i];
  }
  if (sorted && h->n > 0)
    CK(cudaMemcpy(sorted, h->mb.xs, (size_t)h->n * sizeof(double4), cudaMemcpyDeviceToHost));
  return TREE_GPU_OK;
}

int tree_gpu_set_stream(tree_gpu_handle* h, void* stream) {
  if (!h) return TREE_GPU_ERR_ARG;
  CK(cudaStreamSynchronize(h->st));
  h->st = stream ? (cudaStream_t)stream : h->own_st;
  return TREE_GPU_OK;
}

int tree_gpu_set_tuning(tree_gpu_handle* h, int32_t bucket,
                        int32_t blocks_per_sm, int32_t order) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (bucket < 1 || bucket > 8 || blocks_per_sm < 1 || blocks_per_sm > 4 ||
      order < 2 || order > 4)
    return fail(h, TREE_GPU_ERR_ARG,
                "bucket must be 1..8, blocks_per_sm 1..4, order 2..4");
  h->tune.bucket = bucket;
  h->tune.blocks_per_sm = blocks_per_sm;
  h->tune.order = order;
  ++h->epoch;
  return TREE_GPU_OK;
}

int tree_gpu_set_local_expansion(tree_gpu_handle* h, double max_ratio) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (!(max_ratio >= 0.0 && max_ratio <= 0.5))
    return fail(h, TREE_GPU_ERR_ARG, "max_ratio must be in [0, 0.5]");
  h->tune.loc_eps = (float)max_ratio;
  ++h->epoch;
  return TREE_GPU_OK;
}

int tree_gpu_timings(tree_gpu_handle* h, tree_gpu_timing* out) {
  if (!h || !out) return TREE_GPU_ERR_ARG;
  *out = h->timing;
  return TREE_GPU_OK;
}

const char* tree_gpu_last_error(tree_gpu_handle* h) {
  return h ? h->last_error.c_str() : "null handle";
}

int tree_gpu_destroy(tree_gpu_handle* h) {
  if (!h) return TREE_GPU_OK;
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->own_st && h->own_st != h->st) cudaStreamSynchronize(h->own_st);
  free_graphs(h);
  free_all(h);
  for (auto& es : h->events)
    for (int k = 0; k < 4; ++k) cudaEventDestroy(es.e[k]);
  if (h->h_pinned) cudaFreeHost(h->h_pinned);
  if (h->own_st) cudaStreamDestroy(h->own_st);
  delete h;
  return TREE_GPU_OK;
}

const char* tree_gpu_version(void) { return TREE_GPU_VERSION_STR; }

/* ---- ensembles of independent clouds ---- */

int tree_gpu_ensemble_create(const tree_gpu_params* params, int32_t ncloud,
                             const int64_t* n_el, const int64_t* n_ion,
                             tree_gpu_handle** out) {
  if (!out) return TREE_GPU_ERR_ARG;
  *out = nullptr;
  if (!params || !n_el || !n_ion || ncloud < 1 || ncloud > kMaxClouds)
    return TREE_GPU_ERR_ARG;
  int64_t total = 0, total_el = 0;
  for (int c = 0; c < ncloud; ++c) {
    if (check_params(&params[c]) != TREE_GPU_OK) return TREE_GPU_ERR_ARG;
    const tree_gpu_params& a = params[c];
    const tree_gpu_params& p0 = params[0];
    // one walk, one integrator and one criterion for all clouds
    if (a.precision != TREE_GPU_PREC_MIXED || a.physics != p0.physics ||
        a.theta != p0.theta || a.mac != p0.mac || a.xm_el != p0.xm_el ||
        a.xm_ion != p0.xm_ion)
      return TREE_GPU_ERR_ARG;
    if (n_el[c] < 0 || n_ion[c] < 0) return TREE_GPU_ERR_ARG;
    total += n_el[c] + n_ion[c];
    total_el += n_el[c];
  }
  if (total > (int64_t)0x7fffffff / 4) return TREE_GPU_ERR_ARG;
  tree_gpu_handle* h = nullptr;
  int rc = tree_gpu_create(&params[0], total_el, total - total_el, &h);
  if (rc) return rc;
  h->cloud_prm.assign(params, params + ncloud);
  h->cloud_ne.assign(n_el, n_el + ncloud);
  h->cloud_ni.assign(n_ion, n_ion + ncloud);
  std::vector<int32_t> start(ncloud + 1), eend(ncloud);
  std::vector<uint8_t> ion((size_t)std::max<int64_t>(total, 1), 0);
  std::vector<float4> pk(2 * (size_t)ncloud);
  int64_t o = 0;
  for (int c = 0; c < ncloud; ++c) {
    start[c] = (int32_t)o;
    eend[c] = (int32_t)(o + n_el[c]);
    for (int64_t i = o + n_el[c]; i < o + n_el[c] + n_ion[c]; ++i) ion[i] = 1;
    o += n_el[c] + n_ion[c];
    const tree_gpu_params& a = params[c];
    double lam[3] = {1, 1, 1};
    if (a.te > 0.0 && a.xm_el > 0.0 && a.xm_ion > 0.0) {
      lam[0] = kelbg_lambda_um(a.xm_el / 2.0, a.te);
      lam[1] = kelbg_lambda_um(a.xm_el * a.xm_ion / (a.xm_el + a.xm_ion), a.te);
      lam[2] = kelbg_lambda_um(a.xm_ion / 2.0, a.te);
    }
    const float rs_inv = a.rs > 0.0 ? (float)(1.0 / a.rs) : 0.f;
    pk[2 * c] = make_float4((float)(1.0 / (lam[0] * lam[0])), (float)(1.0 / (lam[1] * lam[1])),
                            (float)(1.0 / (lam[2] * lam[2])), rs_inv);
    pk[2 * c + 1] = make_float4((float)(1.0 / lam[0]), (float)(1.0 / lam[1]),
                                (float)(1.0 / lam[2]), 0.f);
  }
  start[ncloud] = (int32_t)o;
  do {
    tg::BuildBuffers& b = h->b;
    if ((rc = dalloc(h, &b.bbox, 6 * (size_t)std::max(2, ncloud)))) break;
    if ((rc = dalloc(h, &b.geom, (size_t)std::max(2, ncloud)))) break;
    if ((rc = dalloc(h, &h->ens_start, (size_t)ncloud + 1))) break;
    if ((rc = dalloc(h, &h->ens_elec_end, (size_t)ncloud))) break;
    if ((rc = dalloc(h, &h->ens_roots, (size_t)ncloud))) break;
    if ((rc = dalloc(h, &h->ens_glvl, (size_t)ncloud * tg::kLevelSlots))) break;
    if ((rc = dalloc(h, &h->cloud_pk, 2 * (size_t)ncloud))) break;
    if ((rc = dalloc(h, &h->ion_flag, ion.size()))) break;
    if ((rc = dalloc(h, &h->cloud_sums, 6 * (size_t)ncloud))) break;
    cudaMemcpy(h->ens_start, start.data(), start.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    cudaMemcpy(h->ens_elec_end, eend.data(), eend.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    cudaMemcpy(h->cloud_pk, pk.data(), pk.size() * sizeof(float4), cudaMemcpyHostToDevice);
    if (cudaMemcpy(h->ion_flag, ion.data(), ion.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "ensemble upload failed");
      break;
    }
    int top = 1;
    while ((1 << top) < ncloud) ++top;
    b.ens.nseg = ncloud;
    b.ens.top = top;
    b.ens.nlev = (126 - top) / 3;
    b.ens.start = h->ens_start;
    b.ens.elec_end = h->ens_elec_end;
    b.ens.roots = h->ens_roots;
    b.ens.glvl = h->ens_glvl;
    ++h->epoch;
  } while (0);
  if (rc) {
    tree_gpu_destroy(h);
    return rc;
  }
  *out = h;
  return TREE_GPU_OK;
}

int tree_gpu_ensemble_load_state(tree_gpu_handle* h, const double* x,
                                 const double* v, const double* f) {
  if (!h || h->b.ens.nseg == 0) return TREE_GPU_ERR_ARG;
  if (h->n && (!x || !v)) return fail(h, TREE_GPU_ERR_ARG, "null particle buffer");
  const size_t bytes = 3 * sizeof(double) * (size_t)h->n;
  if (bytes) {
    CK(cudaMemcpyAsync(h->x, x, bytes, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->v, v, bytes, cudaMemcpyHostToDevice, h->st));
    if (f) CK(cudaMemcpyAsync(h->f, f, bytes, cudaMemcpyHostToDevice, h->st));
  }
  h->nloop = 0;
  if (f) {
    h->has_state = true;
    h->has_fprev = true;
    return TREE_GPU_OK;
  }
  h->has_fprev = false;  // initial forces with the fixed-theta test
  int rc = force_device(h, false);
  if (rc) return rc;
  h->has_state = true;
  h->has_fprev = true;
  return TREE_GPU_OK;
}

int tree_gpu_ensemble_set_state(tree_gpu_handle* h, const double* x, const double* v) {
  return tree_gpu_ensemble_load_state(h, x, v, nullptr);
}

int tree_gpu_ensemble_get_state(tree_gpu_handle* h, double* x, double* v, double* f) {
  if (!h || h->b.ens.nseg == 0) return TREE_GPU_ERR_ARG;
  const size_t bytes = 3 * sizeof(double) * (size_t)h->n;
  if (bytes) {
    if (x) CK(cudaMemcpyAsync(x, h->x, bytes, cudaMemcpyDeviceToHost, h->st));
    if (v) CK(cudaMemcpyAsync(v, h->v, bytes, cudaMemcpyDeviceToHost, h->st));
    if (f) CK(cudaMemcpyAsync(f, h->f, bytes, cudaMemcpyDeviceToHost, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return TREE_GPU_OK;
}

int tree_gpu_ensemble_sums(tree_gpu_handle* h, double* out) {
  if (!h || h->b.ens.nseg == 0 || !out) return TREE_GPU_ERR_ARG;
  const int nc = h->b.ens.nseg;
  tg::cloud_sums(h->x, h->v, h->epot_part, h->ens_start, h->ens_elec_end, nc,
                 h->prm.xm_el, h->prm.xm_ion, h->cloud_sums, h->st);
  h->timing.launches += 1;
  CK(cudaMemcpyAsync(out, h->cloud_sums, 6 * sizeof(double) * nc,
                     cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return TREE_GPU_OK;
}

int tree_gpu_ensemble_direct(tree_gpu_handle* h, int32_t cloud,
                             const int64_t* targets, int64_t nt, double* f,
                             double* epot) {
  if (!h || h->b.ens.nseg == 0) return TREE_GPU_ERR_ARG;
  if (cloud < 0 || cloud >= h->b.ens.nseg) return fail(h, TREE_GPU_ERR_ARG, "cloud index");
  const int64_t ne = h->cloud_ne[cloud], nc = ne + h->cloud_ni[cloud];
  int64_t off = 0;
  for (int c = 0; c < cloud; ++c) off += h->cloud_ne[c] + h->cloud_ni[c];
  if (nt < 0 || nt > 0x7fffffff || (nt && (!targets || !f || !epot)))
    return fail(h, TREE_GPU_ERR_ARG, "bad target list");
  if (nt == 0) return TREE_GPU_OK;
  for (int64_t i = 0; i < nt; ++i)
    if (targets[i] < 0 || targets[i] >= nc)
      return fail(h, TREE_GPU_ERR_ARG, "target index out of range");
  const tree_gpu_params& a = h->cloud_prm[cloud];
  tg::WalkParams wp;
  wp.physics = a.physics;
  wp.theta = a.theta;
  wp.rs = a.rs;
  wp.lam_ee = kelbg_lambda_um(a.xm_el / 2.0, a.te);
  wp.lam_ei = kelbg_lambda_um(a.xm_el * a.xm_ion / (a.xm_el + a.xm_ion), a.te);
  wp.lam_ii = kelbg_lambda_um(a.xm_ion / 2.0, a.te);
  wp.dx_ei = a.dx_ei;
  wp.dx_ii = a.dx_ii;
  int nch = tg::direct_chunks((int)nc, (int)nt);
  int64_t* d_t = nullptr;
  double4* d_part = nullptr;
  double *d_f = nullptr, *d_e = nullptr;
  int rc = TREE_GPU_OK;
  do {
    if (cudaMalloc(&d_t, nt * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&d_part, (size_t)nch * nt * sizeof(double4)) != cudaSuccess ||
        cudaMalloc(&d_f, 3 * nt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_e, nt * sizeof(double)) != cudaSuccess) {
      rc = fail(h, TREE_GPU_ERR_CUDA, "direct-sum scratch allocation failed");
      break;
    }
    cudaMemcpyAsync(d_t, targets, nt * sizeof(int64_t), cudaMemcpyHostToDevice, h->st);
    h->timing.launches += tg::direct_sum(h->x + 3 * off, (int)nc, (int)ne, d_t, (int)nt,
                                         wp, nch, d_part, d_f, d_e, h->st);
    cudaMemcpyAsync(f, d_f, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    cudaMemcpyAsync(epot, d_e, nt * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) rc = fail(h, TREE_GPU_ERR_CUDA, cudaGetErrorString(e));
  } while (0);
  cudaFree(d_t);
  cudaFree(d_part);
  cudaFree(d_f);
  cudaFree(d_e);
  return rc;
}


}  // extern "C"

// ------------------------------------------------------- learned MAC ----
namespace {

int ensure_model_buffers(tree_gpu_handle* h) {
  if (h->mlp_params) return TREE_GPU_OK;
  CK(cudaMalloc(&h->mlp_params, sizeof(float) * tg::kMlpParams));
  CK(cudaMalloc(&h->mlp_stats, sizeof(float) * TREE_GPU_MLP_STATS));
  CK(cudaMalloc(&h->mlp_packed, sizeof(tg::MlpPacked)));
  return TREE_GPU_OK;
}

}  // namespace

extern "C" {

int tree_gpu_mac_collect(tree_gpu_handle* h, double theta_lo, double theta_hi,
                         double rho_lo, double rho_hi, int32_t max_count,
                         float keep, uint64_t seed, int64_t cap,
                         int64_t* n_total) {
  if (h && h->b.ens.nseg > 0)
    return fail(h, TREE_GPU_ERR_ARG, "ensemble handle: use the tree_gpu_ensemble_* calls");
  if (!h) return TREE_GPU_ERR_ARG;
  if (!(theta_lo > 0 && theta_hi >= theta_lo && rho_lo > 0 && rho_hi >= rho_lo) ||
      cap <= 0 || cap > (int64_t)0x7fffffff || max_count < 2 || !(keep > 0.f && keep <= 1.f))
    return fail(h, TREE_GPU_ERR_ARG, "bad sampling arguments");
  if (h->n == 0) return fail(h, TREE_GPU_ERR_STATE, "no particles");
  if (h->smp_cap != cap) {
    if (h->smp_feats) cudaFree(h->smp_feats);
    if (h->smp_labels) cudaFree(h->smp_labels);
    if (h->smp_extra) cudaFree(h->smp_extra);
    if (h->smp_count) cudaFree(h->smp_count);
    h->smp_feats = h->smp_labels = h->smp_extra = nullptr;
    h->smp_count = nullptr;
    CK(cudaMalloc(&h->smp_feats, sizeof(float) * 16 * (size_t)cap));
    CK(cudaMalloc(&h->smp_labels, sizeof(float) * (size_t)cap));
    CK(cudaMalloc(&h->smp_extra, sizeof(float) * 2 * (size_t)cap));
    CK(cudaMalloc(&h->smp_count, sizeof(int32_t) * 2));
    CK(cudaMemsetAsync(h->smp_count, 0, sizeof(int32_t) * 2, h->st));
    h->smp_cap = cap;
  }
  // combined tree of the current device positions, every FP64 record written
  if (int rc = build_full_records(h)) return rc;
  tg::SampleArgs a;
  a.node_c = h->b.node_c;
  a.mom = h->mb.mom;
  a.mom3 = h->mb.mom3;
  a.geom = h->mb.geom;
  a.m64 = h->mb.m64;
  a.kids = h->mb.kids;
  a.first = h->mb.first;
  a.count = h->mb.count;
  a.xs = h->mb.xs;
  a.groups = h->mb.groups;
  a.n_groups = h->mb.control + 2;
  a.cursor = h->smp_count + 1;
  a.stack = h->mb.stack;
  a.theta_lo = (float)theta_lo;
  a.theta_hi = (float)theta_hi;
  a.rho_lo = (float)rho_lo;
  a.rho_hi = (float)rho_hi;
  a.seed = (uint32_t)(seed ^ (seed >> 32));
  a.max_count = max_count;
  a.keep = keep;
  a.order = h->tune.order;
  a.lam_ei = (float)h->lam[1];
  a.feats = h->smp_feats;
  a.labels = h->smp_labels;
  a.extra = h->smp_extra;
  a.n_out = h->smp_count;
  a.cap = (int)cap;
  a.err = h->b.err;
  h->timing.launches += tg::mac_sample(a, h->mb.grid_warps, h->st);
  CK(cudaGetLastError());
  int32_t cnt = 0;
  CK(cudaMemcpyAsync(&cnt, h->smp_count, sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
  bool grow = false;
  int rc = check_device_status(h, &grow);
  if (rc) return rc;
  if (n_total) *n_total = cnt < cap ? cnt : cap;
  return TREE_GPU_OK;
}

int tree_gpu_mac_samples(tree_gpu_handle* h, float* feats, float* labels,
                         float* extra, int64_t cap, int64_t* n) {
  if (!h) return TREE_GPU_ERR_ARG;
  int32_t cnt = 0;
  if (h->smp_count)
    CK(cudaMemcpy(&cnt, h->smp_count, sizeof(int32_t), cudaMemcpyDeviceToHost));
  int64_t m = cnt < h->smp_cap ? cnt : h->smp_cap;
  if (n) *n = m;
  if (!feats && !labels && !extra) return TREE_GPU_OK;
  if (cap < m) return fail(h, TREE_GPU_ERR_ARG, "buffer too small");
  if (m == 0) return TREE_GPU_OK;
  if (feats) CK(cudaMemcpy(feats, h->smp_feats, sizeof(float) * 16 * m, cudaMemcpyDeviceToHost));
  if (labels) CK(cudaMemcpy(labels, h->smp_labels, sizeof(float) * m, cudaMemcpyDeviceToHost));
  if (extra) CK(cudaMemcpy(extra, h->smp_extra, sizeof(float) * 2 * m, cudaMemcpyDeviceToHost));
  return TREE_GPU_OK;
}

int tree_gpu_mac_clear(tree_gpu_handle* h) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (h->smp_count) CK(cudaMemset(h->smp_count, 0, sizeof(int32_t) * 2));
  return TREE_GPU_OK;
}

int tree_gpu_mac_train(tree_gpu_handle* h, int32_t epochs, int32_t batch,
                       float lr, float tau, uint64_t seed,
                       float* loss_per_epoch) {
  if (!h) return TREE_GPU_ERR_ARG;
  int64_t m = 0;
  int rc = tree_gpu_mac_samples(h, nullptr, nullptr, nullptr, 0, &m);
  if (rc) return rc;
  if (m < 64) return fail(h, TREE_GPU_ERR_STATE, "collect samples first");
  if (epochs <= 0 || batch <= 0 || !(lr > 0) || !(tau > 0 && tau < 1))
    return fail(h, TREE_GPU_ERR_ARG, "bad training arguments");
  if ((rc = ensure_model_buffers(h))) return rc;
  int e = tg::mlp_train(h->smp_feats, h->smp_labels, (int)m, epochs, batch, lr,
                        tau, seed, h->mlp_params, h->mlp_stats, loss_per_epoch,
                        h->st);
  if (e) return fail(h, TREE_GPU_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
  h->timing.launches += tg::mlp_pack(h->mlp_params, h->mlp_stats, h->mlp_stats + 16,
                                     h->mlp_packed, h->st);
  CK(cudaStreamSynchronize(h->st));
  h->has_model = true;
  ++h->epoch;
  return TREE_GPU_OK;
}

int tree_gpu_mac_set_model(tree_gpu_handle* h, const float* params,
                           const float* stats) {
  if (!h || !params || !stats) return TREE_GPU_ERR_ARG;
  int rc = ensure_model_buffers(h);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->mlp_params, params, sizeof(float) * tg::kMlpParams,
                     cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->mlp_stats, stats, sizeof(float) * TREE_GPU_MLP_STATS,
                     cudaMemcpyHostToDevice, h->st));
  h->timing.launches += tg::mlp_pack(h->mlp_params, h->mlp_stats, h->mlp_stats + 16,
                                     h->mlp_packed, h->st);
  CK(cudaStreamSynchronize(h->st));
  h->has_model = true;
  ++h->epoch;
  return TREE_GPU_OK;
}

int tree_gpu_mac_get_model(tree_gpu_handle* h, float* params, float* stats) {
  if (!h || !params || !stats) return TREE_GPU_ERR_ARG;
  if (!h->has_model) return fail(h, TREE_GPU_ERR_STATE, "no model");
  CK(cudaMemcpy(params, h->mlp_params, sizeof(float) * tg::kMlpParams, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(stats, h->mlp_stats, sizeof(float) * TREE_GPU_MLP_STATS,
                cudaMemcpyDeviceToHost));
  return TREE_GPU_OK;
}

int tree_gpu_mac_config(tree_gpu_handle* h, float eta, float rho_lo, float rho_hi) {
  if (!h) return TREE_GPU_ERR_ARG;
  if (!(eta > 0) || !(rho_lo > 0) || !(rho_hi >= rho_lo))
    return fail(h, TREE_GPU_ERR_ARG, "bad learned-MAC configuration");
  h->mac_eta = eta;
  ++h->epoch;
  h->mac_rho_lo = rho_lo;
  h->mac_rho_hi = rho_hi;
  return TREE_GPU_OK;
}

int tree_gpu_mlp_grad(const float* X, const float* Y, int64_t n,
                      const float* params, float tau, float* grad, float* loss) {
  if (!X || !Y || !params || !grad || !loss || n <= 0 || n > 0x7fffffff)
    return TREE_GPU_ERR_ARG;
  float *dX = nullptr, *dY = nullptr, *dP = nullptr, *dG = nullptr, *dL = nullptr;
  cudaError_t e = cudaSuccess;
  auto al = [&](float** q, size_t cnt) { if (e == cudaSuccess) e = cudaMalloc(q, cnt * sizeof(float)); };
  al(&dX, 16 * (size_t)n);
  al(&dY, (size_t)n);
  al(&dP, tg::kMlpParams);
  al(&dG, tg::kMlpParams);
  al(&dL, 1);
  if (e == cudaSuccess) {
    cudaMemcpy(dX, X, sizeof(float) * 16 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dY, Y, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dP, params, sizeof(float) * tg::kMlpParams, cudaMemcpyHostToDevice);
    cudaMemset(dG, 0, sizeof(float) * tg::kMlpParams);
    cudaMemset(dL, 0, sizeof(float));
    tg::mlp_grad(dX, dY, (int)n, dP, tau, dG, dL, 64, 0);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
      cudaMemcpy(grad, dG, sizeof(float) * tg::kMlpParams, cudaMemcpyDeviceToHost);
      cudaMemcpy(loss, dL, sizeof(float), cudaMemcpyDeviceToHost);
    }
  }
  float* all[] = {dX, dY, dP, dG, dL};
  for (float* q : all) if (q) cudaFree(q);
  return e == cudaSuccess ? TREE_GPU_OK : TREE_GPU_ERR_CUDA;
}

int tree_gpu_mlp_infer(const float* X, int64_t n, const float* params,
                       const float* stats, float* y) {
  if (!X || !params || !stats || !y || n <= 0 || n > 0x7fffffff) return TREE_GPU_ERR_ARG;
  float *dX = nullptr, *dP = nullptr, *dS = nullptr, *dY = nullptr;
  tg::MlpPacked* dK = nullptr;
  cudaError_t e = cudaSuccess;
  auto al = [&](float** q, size_t cnt) { if (e == cudaSuccess) e = cudaMalloc(q, cnt * sizeof(float)); };
  al(&dX, 16 * (size_t)n);
  al(&dP, tg::kMlpParams);
  al(&dS, TREE_GPU_MLP_STATS);
  al(&dY, (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(&dK, sizeof(tg::MlpPacked));
  if (e == cudaSuccess) {
    cudaMemcpy(dX, X, sizeof(float) * 16 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dP, params, sizeof(float) * tg::kMlpParams, cudaMemcpyHostToDevice);
    cudaMemcpy(dS, stats, sizeof(float) * TREE_GPU_MLP_STATS, cudaMemcpyHostToDevice);
    tg::mlp_pack(dP, dS, dS + 16, dK, 0);
    tg::mlp_infer(dX, (int)n, dK, dY, 0);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) cudaMemcpy(y, dY, sizeof(float) * n, cudaMemcpyDeviceToHost);
  }
  float* all[] = {dX, dP, dS, dY};
  for (float* q : all) if (q) cudaFree(q);
  if (dK) cudaFree(dK);
  return e == cudaSuccess ? TREE_GPU_OK : TREE_GPU_ERR_CUDA;
}

}  // extern "C"
