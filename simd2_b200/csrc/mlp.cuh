// mlp.cuh -- the cost model of the learned dispatch: a 12-32-32-1 ReLU MLP
// that predicts log2(time in ms) of one closure step for a kernel
// configuration, with hand-written training and inference kernels.
//
// Input (kMlpIn = 12): seven step features computed on the device from the
// block occupancy statistics (see mlp_features) followed by the configuration
// encoding: one-hot split factor {1,2,4,8} and the skip flag.
// Parameters are one flat float array:
//   W1[H][In] | b1[H] | W2[H][H] | b2[H] | W3[H] | b3
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kMlpIn = 12;
constexpr int kMlpFeat = 7;
constexpr int kMlpH = 32;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpH * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpH;
constexpr int kMlpB2 = kMlpW2 + kMlpH * kMlpH;
constexpr int kMlpW3 = kMlpB2 + kMlpH;
constexpr int kMlpB3 = kMlpW3 + kMlpH;
constexpr int kMlpParams = kMlpB3 + 1;  // 1505
constexpr int kNumConfigs = 8;          // split {1,2,4,8} x skip {0,1}
constexpr int kLearnedMinN = 1024;      // the learned policy runs the plain path up to this n,
constexpr int kLearnedLoopMinN = 2048;  // then a sparse opening, and per-step MLP choices above this n

__host__ __device__ inline int config_split(int c) { return 1 << (c & 3); }
__host__ __device__ inline int config_skip(int c) { return c >> 2; }

__device__ __forceinline__ void mlp_encode_config(int c, float* x /* kMlpIn */) {
  for (int j = 0; j < 4; j++) x[kMlpFeat + j] = (c & 3) == j ? 1.f : 0.f;
  x[kMlpFeat + 4] = (float)config_skip(c);
}

// Forward pass of one sample; z1, z2 receive the pre-activations when non-null.
__device__ float mlp_forward_one(const float* __restrict__ P, const float* x, float* z1, float* z2) {
  float h1[kMlpH];
#pragma unroll 4
  for (int j = 0; j < kMlpH; j++) {
    float s = P[kMlpB1 + j];
    for (int i = 0; i < kMlpIn; i++) s = fmaf(P[kMlpW1 + j * kMlpIn + i], x[i], s);
    if (z1) z1[j] = s;
    h1[j] = fmaxf(s, 0.f);
  }
  float out = P[kMlpB3];
#pragma unroll 4
  for (int j = 0; j < kMlpH; j++) {
    float s = P[kMlpB2 + j];
    for (int i = 0; i < kMlpH; i++) s = fmaf(P[kMlpW2 + j * kMlpH + i], h1[i], s);
    if (z2) z2[j] = s;
    out = fmaf(P[kMlpW3 + j], fmaxf(s, 0.f), out);
  }
  return out;
}

__global__ void mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ X, int B,
                                   float* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    float x[kMlpIn];
    for (int i = 0; i < kMlpIn; i++) x[i] = X[(long long)b * kMlpIn + i];
    out[b] = mlp_forward_one(P, x, nullptr, nullptr);
  }
}

// Per-sample gradient of L = (1/B) sum_b (out_b - y_b)^2, written to G[b][P].
__global__ void mlp_sample_grad_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                       const float* __restrict__ y, int B, float* __restrict__ G) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    float x[kMlpIn], z1[kMlpH], z2[kMlpH];
    for (int i = 0; i < kMlpIn; i++) x[i] = X[(long long)b * kMlpIn + i];
    const float out = mlp_forward_one(P, x, z1, z2);
    const float d_out = 2.f * (out - y[b]) / (float)B;
    float* g = G + (long long)b * kMlpParams;
    g[kMlpB3] = d_out;
    float d1[kMlpH];
    for (int i = 0; i < kMlpH; i++) d1[i] = 0.f;
    for (int j = 0; j < kMlpH; j++) {
      const float a2 = fmaxf(z2[j], 0.f);
      g[kMlpW3 + j] = d_out * a2;
      const float d2 = z2[j] > 0.f ? d_out * P[kMlpW3 + j] : 0.f;
      g[kMlpB2 + j] = d2;
      for (int i = 0; i < kMlpH; i++) {
        g[kMlpW2 + j * kMlpH + i] = d2 * fmaxf(z1[i], 0.f);
        d1[i] = fmaf(d2, P[kMlpW2 + j * kMlpH + i], d1[i]);
      }
    }
    for (int j = 0; j < kMlpH; j++) {
      const float dz = z1[j] > 0.f ? d1[j] : 0.f;
      g[kMlpB1 + j] = dz;
      for (int i = 0; i < kMlpIn; i++) g[kMlpW1 + j * kMlpIn + i] = dz * x[i];
    }
  }
}

// grad[p] = sum_b G[b][p], summed in b order (deterministic).
__global__ void column_sum_kernel(const float* __restrict__ G, int B, int P, float* __restrict__ grad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < B; b++) s += G[(long long)b * P + p];
    grad[p] = s;
  }
}

// Adam (Kingma & Ba 2015) with bias correction; t is the 1-based step.
__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float beta1, float beta2, float eps, int t) {
  const float c1 = 1.f - powf(beta1, (float)t);
  const float c2 = 1.f - powf(beta2, (float)t);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const float g = grad[p];
    const float mm = beta1 * m[p] + (1.f - beta1) * g;
    const float vv = beta2 * v[p] + (1.f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    P[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

// The seven step features from the occupancy statistics
// stats = {surviving (tm,tn,kt) triples, occupied A blocks, occupied B blocks}.
__host__ __device__ inline void mlp_features(int n, int tiles_m, int tiles_n, int ktiles,
                                             unsigned long long triples, unsigned long long occa,
                                             unsigned long long occb, int sms, float* f) {
  const double tiles = (double)tiles_m * tiles_n;
  f[0] = (float)(log2((double)n) / 16.0);
  f[1] = (float)((double)triples / (tiles * ktiles));
  f[2] = (float)((double)occa / ((double)tiles_m * ktiles));
  f[3] = (float)((double)occb / ((double)ktiles * tiles_n));
  f[4] = (float)(log2(tiles) / 16.0);
  f[5] = (float)fmin(tiles / sms, 16.0) / 16.f;
  f[6] = (float)(log2((double)triples + 1.0) / 32.0);
}

// Picks the configuration with the smallest predicted time for one step.
// out[0] = chosen config, out[1..8] = predictions (as float bits).
__global__ void mlp_choose_kernel(const float* __restrict__ P, const unsigned long long* __restrict__ stats, int n,
                                  int tiles_m, int tiles_n, int ktiles, int sms, int allow_skip, int max_split,
                                  int* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float x[kMlpIn];
  mlp_features(n, tiles_m, tiles_n, ktiles, stats[0], stats[1], stats[2], sms, x);
  int best = 0;
  float best_t = 3.0e38f;
  for (int c = 0; c < kNumConfigs; c++) {
    mlp_encode_config(c, x);
    const float t = mlp_forward_one(P, x, nullptr, nullptr);
    out[1 + c] = __float_as_int(t);
    const bool allowed = (allow_skip || !config_skip(c)) && config_split(c) <= max_split;
    if (allowed && t < best_t) {
      best_t = t;
      best = c;
    }
  }
  out[0] = best;
}

}  // namespace simd2
