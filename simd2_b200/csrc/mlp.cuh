// mlp.cuh -- the cost model of the learned dispatch: a 15-32-32-1 ReLU MLP
// that predicts log2(time in ms) of one closure step for a step
// configuration, with hand-written training and inference kernels.
//
// Input (kMlpIn = 15): nine step features computed on the device from the
// block occupancy and the entry counts of X_t (see mlp_features) followed by
// the configuration encoding: one-hot split factor {1,2,4,8}, the skip flag
// and the sparse flag (a CSR SpGEMM step, configuration kSparseConfig).
// Parameters are one flat float array:
//   W1[H][In] | b1[H] | W2[H][H] | b2[H] | W3[H] | b3
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kMlpIn = 15;
constexpr int kMlpFeat = 9;
constexpr int kMlpH = 32;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpH * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpH;
constexpr int kMlpB2 = kMlpW2 + kMlpH * kMlpH;
constexpr int kMlpW3 = kMlpB2 + kMlpH;
constexpr int kMlpB3 = kMlpW3 + kMlpH;
constexpr int kMlpParams = kMlpB3 + 1;  // 1601
constexpr int kNumConfigs = 8;          // dense: split {1,2,4,8} x skip {0,1}
constexpr int kSparseConfig = 8;        // a CSR SpGEMM step
constexpr int kLearnedMinN = 1024;      // the learned policy runs the plain path up to this n,
constexpr int kLearnedLoopMinN = 2048;  // then a sparse opening, and per-step MLP choices above this n

__host__ __device__ inline int config_split(int c) { return 1 << (c & 3); }
__host__ __device__ inline int config_skip(int c) { return c >> 2; }

__device__ __forceinline__ void mlp_encode_config(int c, float* x /* kMlpIn */) {
  const bool sparse = c == kSparseConfig;
  for (int j = 0; j < 4; j++) x[kMlpFeat + j] = !sparse && (c & 3) == j ? 1.f : 0.f;
  x[kMlpFeat + 4] = sparse ? 0.f : (float)config_skip(c);
  x[kMlpFeat + 5] = sparse ? 1.f : 0.f;
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

// The nine step features from the statistics of X_t:
// stats = {surviving (tm,tn,kt) triples, occupied A panels, occupied B
// panels, stored entries, Gustavson products sum_k rowcnt(k) colcnt(k)}.
__host__ __device__ inline void mlp_features(int n, int tiles_m, int tiles_n, int ktiles,
                                             const unsigned long long* st, int sms, float* f) {
  const double tiles = (double)tiles_m * tiles_n;
  const double ln = log2((double)n);
  f[0] = (float)(ln / 16.0);
  f[1] = (float)((double)st[0] / (tiles * ktiles));
  f[2] = (float)((double)st[1] / ((double)tiles_m * ktiles));
  f[3] = (float)((double)st[2] / ((double)ktiles * tiles_n));
  f[4] = (float)(log2(tiles) / 16.0);
  f[5] = (float)fmin(tiles / sms, 16.0) / 16.f;
  f[6] = (float)(log2((double)st[0] + 1.0) / 32.0);
  f[7] = (float)((double)st[3] / ((double)n * n));
  f[8] = (float)(log2((double)st[4] + 1.0) / (3.0 * ln));
}

// Picks the configuration with the smallest predicted time for one step:
// the dense ones allowed by allow_skip / max_split, and the sparse step when
// allow_sparse.  Thread c evaluates configuration c; out[0] = chosen config
// (the lowest id among equal predictions), out[1 + c] = prediction for
// config c (as float bits), c = 0..kSparseConfig.  Launch with 32 threads.
__global__ void mlp_choose_kernel(const float* __restrict__ P, const unsigned long long* __restrict__ stats, int n,
                                  int tiles_m, int tiles_n, int ktiles, int sms, int allow_skip, int max_split,
                                  int allow_sparse, int* __restrict__ out) {
  const int c = threadIdx.x;
  float t = 3.0e38f;
  if (blockIdx.x == 0 && c <= kSparseConfig) {
    unsigned long long st[5];
    for (int i = 0; i < 5; i++) st[i] = stats[i];
    float x[kMlpIn];
    mlp_features(n, tiles_m, tiles_n, ktiles, st, sms, x);
    mlp_encode_config(c, x);
    const float p = mlp_forward_one(P, x, nullptr, nullptr);
    out[1 + c] = __float_as_int(p);
    const bool allowed = c == kSparseConfig ? allow_sparse != 0
                                            : (allow_skip || !config_skip(c)) && config_split(c) <= max_split;
    if (allowed) t = p;
  }
  // argmin over the lanes, lower config id on ties
  int best = c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float t2 = __shfl_xor_sync(0xffffffffu, t, o);
    const int b2 = __shfl_xor_sync(0xffffffffu, best, o);
    if (t2 < t || (t2 == t && b2 < best)) {
      t = t2;
      best = b2;
    }
  }
  if (blockIdx.x == 0 && c == 0) out[0] = t < 3.0e38f ? best : 0;
}

}  // namespace simd2
