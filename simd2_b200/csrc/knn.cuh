// knn.cuh -- k-nearest-neighbour tail of the PLD app: the k smallest squared
// distances of every row of a distance block, with their column indices, then
// their square roots.  Restates apps/pld/emulation/knncuda.cu:171-238
// (modified insertion sort + compute_sqrt): among equal distances the lower
// reference index comes first, exactly the order the insertion sort keeps.
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kKnnMaxK = 32;

// Insert (v, i) into an ascending list of K (strictly smaller goes ahead,
// so the earlier index of equal distances stays first).
template <int K>
__device__ __forceinline__ void topk_insert(float (&bd)[K], int (&bi)[K], float v, int i) {
  // Position t takes bd[t-1] when that is larger than v (shift right), else v
  // when bd[t] is larger than v (the insertion point), else keeps bd[t].
  // Every index is a compile-time constant, so the lists stay in registers.
#pragma unroll
  for (int t = K - 1; t > 0; t--) {
    const bool shift = bd[t - 1] > v;
    const bool place = !shift && bd[t] > v;
    bd[t] = shift ? bd[t - 1] : (place ? v : bd[t]);
    bi[t] = shift ? bi[t - 1] : (place ? i : bi[t]);
  }
  if (bd[0] > v) {
    bd[0] = v;
    bi[0] = i;
  }
}

// Lexicographic (distance, index) order.
__device__ __forceinline__ bool lex_less(float a, int ia, float b, int ib) { return a < b || (a == b && ia < ib); }

// One block (kKnnWarps warps) per row.  Warp w scans its contiguous segment
// of the row with 16-byte loads (two in flight per lane); each lane keeps the
// K smallest of its elements, which it visits in increasing index order.  The
// lanes' lists are merged per warp into shared memory, and warp 0 merges the
// warps' lists, all by (distance, index); then the K survivors (and their
// square roots) are written.
constexpr int kKnnWarps = 8;

template <int K>
__global__ void __launch_bounds__(kKnnWarps * 32)
    knn_topk_kernel(const float* __restrict__ dist, long long ldd, int rows, int cols, int col_base,
                    float* __restrict__ out_d, int32_t* __restrict__ out_i, long long ldo, int kout, int take_sqrt) {
  __shared__ float s_d[kKnnWarps][K];
  __shared__ int s_i[kKnnWarps][K];
  __shared__ float s_scr[8][kKnnWarps * 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float inf = __int_as_float(0x7f800000);
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    float bd[K];
    int bi[K];
#pragma unroll
    for (int t = 0; t < K; t++) {
      bd[t] = inf;
      bi[t] = 0x7fffffff;
    }
    const float* row = dist + (long long)r * ldd;
    // segment of this warp, a multiple of 4 elements long
    const int seg = ((cols + kKnnWarps - 1) / kKnnWarps + 3) & ~3;
    const int c0 = warp * seg, c1 = min(cols, c0 + seg);
    const bool vec = ((ldd & 3) == 0) && ((reinterpret_cast<uintptr_t>(dist) & 15) == 0);
    if (vec) {
      // 128 elements per warp per step: lane owns c0 + 128 s + 4 lane .. +3
      for (int c = c0 + 4 * lane; c < c1; c += 256) {
        float4 v0 = make_float4(inf, inf, inf, inf), v1 = v0;
        if (c + 3 < c1) v0 = *reinterpret_cast<const float4*>(row + c);
        else {
          v0.x = c < c1 ? row[c] : inf;
          v0.y = c + 1 < c1 ? row[c + 1] : inf;
          v0.z = c + 2 < c1 ? row[c + 2] : inf;
        }
        const int d = c + 128;
        if (d + 3 < c1) v1 = *reinterpret_cast<const float4*>(row + d);
        else if (d < c1) {
          v1.x = row[d];
          v1.y = d + 1 < c1 ? row[d + 1] : inf;
          v1.z = d + 2 < c1 ? row[d + 2] : inf;
        }
        const float vals[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
        uint32_t mask = 0;
#pragma unroll
        for (int u = 0; u < 8; u++) mask |= (vals[u] < bd[K - 1] ? 1u : 0u) << u;
        if (mask) {
          // one copy of the insertion code; the values go through this
          // thread's shared-memory column for indexed access
#pragma unroll
          for (int u = 0; u < 8; u++) s_scr[u][threadIdx.x] = vals[u];
          do {
            const int u = __ffs(mask) - 1;
            mask &= mask - 1;
            const float v = s_scr[u][threadIdx.x];
            if (v < bd[K - 1]) topk_insert<K>(bd, bi, v, col_base + (u < 4 ? c : d) + (u & 3));
          } while (mask);
        }
      }
    } else {
      for (int c = c0 + lane; c < c1; c += 32) {
        const float v = row[c];
        if (v < bd[K - 1]) topk_insert<K>(bd, bi, v, col_base + c);
      }
    }
    // warp merge of the lanes' heads, K rounds
    int head = 0;
    for (int t = 0; t < K; t++) {
      float v = head < K ? bd[0] : inf;
      int ix = head < K ? bi[0] : 0x7fffffff;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, ix, o);
        if (lex_less(v2, i2, v, ix)) {
          v = v2;
          ix = i2;
        }
      }
      if (head < K && bd[0] == v && bi[0] == ix) {
#pragma unroll
        for (int u = 0; u < K - 1; u++) {
          bd[u] = bd[u + 1];
          bi[u] = bi[u + 1];
        }
        bd[K - 1] = inf;
        bi[K - 1] = 0x7fffffff;
        head++;
      }
      if (lane == 0) {
        s_d[warp][t] = v;
        s_i[warp][t] = ix;
      }
    }
    __syncthreads();
    if (warp == 0) {
      // lane w < kKnnWarps walks warp w's sorted list
      int pos = 0;
      for (int t = 0; t < K; t++) {
        float v = (lane < kKnnWarps && pos < K) ? s_d[lane][pos] : inf;
        int ix = (lane < kKnnWarps && pos < K) ? s_i[lane][pos] : 0x7fffffff;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
          const int i2 = __shfl_xor_sync(0xffffffffu, ix, o);
          if (lex_less(v2, i2, v, ix)) {
            v = v2;
            ix = i2;
          }
        }
        if (lane < kKnnWarps && pos < K && s_d[lane][pos] == v && s_i[lane][pos] == ix) pos++;
        if (lane == 0 && t < kout) {
          out_d[(long long)r * ldo + t] = take_sqrt ? sqrtf(fmaxf(v, 0.f)) : v;
          out_i[(long long)r * ldo + t] = ix == 0x7fffffff ? -1 : ix;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace simd2
