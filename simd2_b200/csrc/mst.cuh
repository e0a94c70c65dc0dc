// mst.cuh -- minimum spanning forest from the min_max closure.
//
// The reference's mst app (apps/mst/cuASR/mst_cuASR.cu) computes the minimax
// (bottleneck) closure D[u][v] = min over paths of the largest edge weight,
// with cuasr_minmax_srsgemm, and stops there.  The spanning forest follows
// from D: order the edges totally by (weight, u, v); an edge of the unique
// minimum spanning forest under that order has no u-v path of smaller edges,
// so its weight equals D[u][v].  The edges with w(u, v) == D[u][v] therefore
// contain the forest, and Kruskal over just those candidates (a handful per
// vertex; all equal-weight alternatives) returns exactly the forest Kruskal
// returns over all edges.  The candidate scan runs on the GPU, the union-find
// on the host.
#pragma once
#include "common.cuh"

namespace simd2 {

// S[i][j] = min(W[i][j], W[j][i]) off the diagonal, 0 on it: the undirected
// weights (+inf where neither direction has an edge).
__global__ void mst_symmetrize_kernel(int n, const float* __restrict__ W, long long ldw, float* __restrict__ S) {
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    const float a = W[(long long)i * ldw + j], b = W[(long long)j * ldw + i];
    S[t] = i == j ? 0.f : ((b < a) ? b : a);
  }
}

// Candidate edges u < v with a finite weight equal to the closed minimax
// value.  COUNT: *count only; otherwise (u, v, w) at atomically taken slots
// below cap.
template <bool COUNT>
__global__ void mst_candidates_kernel(int n, const float* __restrict__ S, const float* __restrict__ D,
                                      int* __restrict__ count, int cap, int* __restrict__ uv,
                                      float* __restrict__ w) {
  const long long total = (long long)n * n;
  const float inf = __int_as_float(0x7f800000);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    if (j <= i) continue;
    const float s = S[t];
    if (!(s < inf) || __float_as_uint(s) != __float_as_uint(D[t])) continue;
    const int slot = atomicAdd(count, 1);
    if (!COUNT && slot < cap) {
      uv[2 * slot] = i;
      uv[2 * slot + 1] = j;
      w[slot] = s;
    }
  }
}

}  // namespace simd2
