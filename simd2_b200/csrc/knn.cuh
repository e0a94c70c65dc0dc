// knn.cuh -- k-nearest-neighbour tail of the PLD app: the k smallest squared
// distances of every row of a distance block, with their column indices, then
// their square roots.  Restates apps/pld/emulation/knncuda.cu:171-238
// (modified insertion sort + compute_sqrt): among equal distances the lower
// reference index comes first, exactly the order the insertion sort keeps.
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kKnnMaxK = 32;

// One warp per row.  Each lane keeps a sorted list of the K smallest
// (distance, index) pairs of columns lane, lane+32, ... (strictly-smaller
// insertion, so the first of equal distances stays ahead); the warp then
// extracts the K overall smallest by repeated (distance, index) arg-min.
template <int K>
__global__ void knn_topk_kernel(const float* __restrict__ dist, long long ldd, int rows, int cols, int col_base,
                                float* __restrict__ out_d, int32_t* __restrict__ out_i, long long ldo, int kout,
                                int take_sqrt) {
  const int warps = blockDim.x / 32;
  const int lane = threadIdx.x & 31;
  for (int r = blockIdx.x * warps + threadIdx.x / 32; r < rows; r += gridDim.x * warps) {
    float bd[K];
    int bi[K];
#pragma unroll
    for (int t = 0; t < K; t++) {
      bd[t] = __int_as_float(0x7f800000);
      bi[t] = 0x7fffffff;
    }
    const float* row = dist + (long long)r * ldd;
    for (int c = lane; c < cols; c += 32) {
      const float v = row[c];
      if (v < bd[K - 1]) {
        // insert keeping ascending order; earlier (lower-index) equal values stay ahead
        int pos = K - 1;
#pragma unroll
        for (int t = K - 1; t > 0; t--) {
          if (pos == t && bd[t - 1] > v) {
            bd[t] = bd[t - 1];
            bi[t] = bi[t - 1];
            pos = t - 1;
          }
        }
        bd[pos] = v;
        bi[pos] = col_base + c;
      }
    }
    // warp merge: K rounds of lexicographic (distance, index) minimum over the lanes' heads
    int head = 0;
    for (int t = 0; t < K; t++) {
      float v = head < K ? bd[0] : __int_as_float(0x7f800000);
      int ix = head < K ? bi[0] : 0x7fffffff;
      for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, ix, o);
        if (v2 < v || (v2 == v && i2 < ix)) {
          v = v2;
          ix = i2;
        }
      }
      // the owner pops its head
      if (head < K && bd[0] == v && bi[0] == ix) {
#pragma unroll
        for (int u = 0; u < K - 1; u++) {
          bd[u] = bd[u + 1];
          bi[u] = bi[u + 1];
        }
        bd[K - 1] = __int_as_float(0x7f800000);
        bi[K - 1] = 0x7fffffff;
        head++;
      }
      if (lane == 0 && t < kout) {
        out_d[(long long)r * ldo + t] = take_sqrt ? sqrtf(fmaxf(v, 0.f)) : v;
        out_i[(long long)r * ldo + t] = ix == 0x7fffffff ? -1 : ix;
      }
    }
  }
}

}  // namespace simd2
