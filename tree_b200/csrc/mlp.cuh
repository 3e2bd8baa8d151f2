// mlp.cuh -- the learned-MAC network on BF16 tensor cores (warp level).
//
// Network: 16 -> 64 -> 64 -> 1, ReLU, layers 1-2 as BF16 mma.sync.m16n8k16
// with FP32 accumulation, layer 3 in FP32.  A warp evaluates 32 samples at a
// time (one per lane).  The walk calls it at warp granularity on the batch of
// cells the warp is testing, so the warp-synchronous mma is the natural unit
// (a CTA-wide tcgen05 tile would need 128 rows that one group never has).
//
// Flat FP32 parameter layout (tree_gpu.h, oracle/mlp.py):
//   W1[16][64] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3[1]
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace tg {

constexpr int kMlpIn = 16;
constexpr int kMlpH = 64;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpIn * kMlpH;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH;
constexpr int kMlpParams = kOffB3 + 1;  // 5313

// Packed inference weights (built by k_mlp_pack from the FP32 parameters):
//   w1f: B fragments of W1, [nt 8][lane 32] x uint2      (2 KB)
//   w2f: B fragments of W2, [kt 4][nt 8][lane 32] x uint2 (8 KB)
//   vec: b1[64] | b2[64] | w3[64] | b3 | feature mean[16] | feature 1/std[16]
constexpr int kMlpVec = 3 * kMlpH + 1 + 2 * kMlpIn;  // 225 floats
struct MlpPacked {
  uint2 w1f[8 * 32];
  uint2 w2f[4 * 8 * 32];
  float vec[kMlpVec + 3];  // padded to a multiple of 4
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// D = A(16x16, row) * B(16x8, col) + C, BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4],
                                               const uint32_t b[2],
                                               const float c[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%10,%11,%12,%13};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]),
        "f"(c[0]), "f"(c[1]), "f"(c[2]), "f"(c[3]));
}

// A fragment (16x16 tile at rows m0.., cols k0..) of a matrix in FP32 shared
// memory with element (m, k) at buf[m*sm + k*sk], optionally ReLU'd.
template <bool RELU>
__device__ __forceinline__ void load_a_f32(uint32_t a[4], const float* buf,
                                           int sm, int sk, int m0, int k0,
                                           int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int r0 = m0 + g, r1 = m0 + g + 8;
  const int c0 = k0 + 2 * t, c1 = k0 + 2 * t + 8;
  auto v = [&](int m, int k) {
    float x = buf[m * sm + k * sk];
    return RELU ? fmaxf(x, 0.f) : x;
  };
  a[0] = pack_bf16x2(v(r0, c0), v(r0, c0 + 1));
  a[1] = pack_bf16x2(v(r1, c0), v(r1, c0 + 1));
  a[2] = pack_bf16x2(v(r0, c1), v(r0, c1 + 1));
  a[3] = pack_bf16x2(v(r1, c1), v(r1, c1 + 1));
}

// B fragment (16x8 tile at rows k0.., cols n0..) of a matrix in FP32 shared
// memory with element (k, n) at buf[k*sk + n*sn].
__device__ __forceinline__ void load_b_f32(uint32_t b[2], const float* buf,
                                           int sk, int sn, int k0, int n0,
                                           int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int n = n0 + g, k = k0 + 2 * t;
  b[0] = pack_bf16x2(buf[k * sk + n * sn], buf[(k + 1) * sk + n * sn]);
  b[1] = pack_bf16x2(buf[(k + 8) * sk + n * sn], buf[(k + 9) * sk + n * sn]);
}

// Inference for the 32 lanes' feature vectors.  xs_tile: 32x16 FP32
// per-warp scratch whose row `lane` holds this lane's raw features on entry
// (normalised in place); P: packed weights in shared memory.  Returns this
// lane's prediction.  All 32 lanes must call it.
// The hidden layer never leaves registers: the accumulator fragment of two
// adjacent 16x8 output tiles of layer 1 (rows g, g+8; columns 2t, 2t+1 of each
// tile) is exactly the A fragment of one 16x16 k-tile of layer 2, so H1 is
// rounded to BF16 and packed in place.
__device__ __forceinline__ float mlp_forward_warp(float* xs_tile,
                                                  const MlpPacked& P,
                                                  int lane) {
  const float* b1 = P.vec;
  const float* b2 = P.vec + kMlpH;
  const float* w3 = P.vec + 2 * kMlpH;
  const float b3 = P.vec[3 * kMlpH];
  const float* mu = P.vec + 3 * kMlpH + 1;
  const float* isd = mu + kMlpIn;
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k)
    xs_tile[lane * kMlpIn + k] = (xs_tile[lane * kMlpIn + k] - mu[k]) * isd[k];
  __syncwarp();
  const int t = lane & 3;
  float part[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [mt][row g / g+8]
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    uint32_t a[4];
    load_a_f32<false>(a, xs_tile, kMlpIn, 1, 16 * mt, 0, lane);
    // layer 1: H1 = relu(X W1 + b1) for rows 16 mt .. 16 mt + 15
    uint32_t h[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const uint2 bb = P.w1f[nt * 32 + lane];
      const uint32_t b[2] = {bb.x, bb.y};
      const float z[4] = {0.f, 0.f, 0.f, 0.f};
      float c[4];
      mma_bf16_16816(c, a, b, z);
      const int col = 8 * nt + 2 * t;
      const uint32_t lo = pack_bf16x2(fmaxf(c[0] + b1[col], 0.f), fmaxf(c[1] + b1[col + 1], 0.f));
      const uint32_t hi = pack_bf16x2(fmaxf(c[2] + b1[col], 0.f), fmaxf(c[3] + b1[col + 1], 0.f));
      h[nt >> 1][(nt & 1) * 2] = lo;
      h[nt >> 1][(nt & 1) * 2 + 1] = hi;
    }
    // layers 2 + 3: y = relu(H1 W2 + b2) . w3 + b3, four 16x8 output tiles
    // at a time so that four independent mma chains overlap
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      float c[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
      for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint2 bb = P.w2f[(kt * 8 + 4 * half + j) * 32 + lane];
          const uint32_t b[2] = {bb.x, bb.y};
          mma_bf16_16816(c[j], h[kt], b, c[j]);
        }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int col = 8 * (4 * half + j) + 2 * t;
        part[mt][0] += fmaxf(c[j][0] + b2[col], 0.f) * w3[col] +
                       fmaxf(c[j][1] + b2[col + 1], 0.f) * w3[col + 1];
        part[mt][1] += fmaxf(c[j][2] + b2[col], 0.f) * w3[col] +
                       fmaxf(c[j][3] + b2[col + 1], 0.f) * w3[col + 1];
      }
    }
  }
  // rows are shared by the 4 threads of a quad
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      part[mt][hh] += __shfl_xor_sync(0xffffffffu, part[mt][hh], 1);
      part[mt][hh] += __shfl_xor_sync(0xffffffffu, part[mt][hh], 2);
    }
  // row r = 16 mt + 8 h + g lives in lanes 4g..4g+3
  const int src = 4 * (lane & 7);
  const float y00 = __shfl_sync(0xffffffffu, part[0][0], src);
  const float y01 = __shfl_sync(0xffffffffu, part[0][1], src);
  const float y10 = __shfl_sync(0xffffffffu, part[1][0], src);
  const float y11 = __shfl_sync(0xffffffffu, part[1][1], src);
  const int q = lane >> 3;
  const float y = q == 0 ? y00 : (q == 1 ? y01 : (q == 2 ? y10 : y11));
  __syncwarp();
  return y + b3;
}

}  // namespace tg
