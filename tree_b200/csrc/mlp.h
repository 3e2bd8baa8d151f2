// mlp.h -- host-side entry points of the learned MAC (training, sampling).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "mlp.cuh"

namespace tg {

// Gradient of the mean pinball loss (quantile tau) over n samples; adds into
// grad (kMlpParams floats) and loss (1 float).  Returns kernels launched.
int mlp_grad(const float* X, const float* Y, int n, const float* params,
             float tau, float* grad, float* loss, int blocks, cudaStream_t st);
size_t mlp_grad_smem();
// Adam step t (1-based) on the FP32 parameters; zeroes grad.
int mlp_adam(float* params, float* grad, float* m, float* v, float lr, int t,
             cudaStream_t st);
int mlp_pack(const float* params, const float* mean, const float* inv_std,
             MlpPacked* out, cudaStream_t st);
int mlp_infer(const float* X, int n, const MlpPacked* packed, float* y,
              cudaStream_t st);

// Trains from scratch on n device samples (raw features X, labels Y):
// computes the feature statistics into stats (72 floats: mean, 1/std, min,
// max, then the 1% and 99% quantiles of label minus feature 15), shuffles, runs `epochs` of Adam with mini-batches of `batch` and a
// cosine learning-rate decay, and leaves the parameters in params.  Returns
// 0 or a CUDA error code; loss_per_epoch (host, may be null) gets the mean
// pinball loss of every epoch.
int mlp_train(const float* X, const float* Y, int n, int epochs, int batch,
              float lr, float tau, uint64_t seed, float* params, float* stats,
              float* loss_per_epoch, cudaStream_t st);

struct SampleArgs {
  const double4* node_c;
  const float4* mom;
  const float4* mom3;
  const float4* geom;
  const double2* m64;
  const int32_t* kids;
  const int32_t* first;
  const int32_t* count;
  const double4* xs;
  const int2* groups;
  const int32_t* n_groups;
  int32_t* cursor;
  int32_t* stack;
  float theta_lo, theta_hi, rho_lo, rho_hi;
  uint32_t seed;
  int max_count;
  float keep;     // probability of keeping a candidate sample
  int order;      // expansion order of the labels (the walk's)
  float lam_ei;
  float* feats;   // cap x 16
  float* labels;  // cap
  float* extra;   // cap x 2: (theta of the walk, rho)
  int32_t* n_out;
  int cap;
  int32_t* err;
};

int mac_sample(const SampleArgs& a, int grid_warps, cudaStream_t st);
int mac_sample_stack_per_warp();

}  // namespace tg
