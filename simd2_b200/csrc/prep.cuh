// prep.cuh -- operand preparation kernels (HBM-bound, one pass each).
#pragma once
#include "common.cuh"

namespace simd2 {

// B'[p][2j+e] = B[2p+e][j] for 2p+e < K and j < N, else `pad`.
// B' has Kp/2 rows of 2*Np floats (Kp, Np are the padded sizes).  Each thread
// writes one float4 = (B[2p][j], B[2p+1][j], B[2p][j+1], B[2p+1][j+1]).
template <typename T, int MODE>
__device__ __forceinline__ float load_operand(const T* p) {
  if constexpr (MODE == 1) return (*p != T(0)) ? 1.0f : 0.0f;  // boolean (or_and as max_min on {0,1})
  else return static_cast<float>(*p);
}

template <typename T, int MODE>
__global__ void interleave_pairs_kernel(const T* __restrict__ B, long long ldb, int K, int N,
                                        float* __restrict__ Bp, int Kp, int Np, float pad) {
  const long long pairs_j = Np / 2;
  const long long total = (long long)(Kp / 2) * pairs_j;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / pairs_j);
    const int j = (int)(t - (long long)p * pairs_j) * 2;
    const int k0 = 2 * p, k1 = 2 * p + 1;
    float4 v;
    v.x = (k0 < K && j < N) ? load_operand<T, MODE>(B + (long long)k0 * ldb + j) : pad;
    v.y = (k1 < K && j < N) ? load_operand<T, MODE>(B + (long long)k1 * ldb + j) : pad;
    v.z = (k0 < K && j + 1 < N) ? load_operand<T, MODE>(B + (long long)k0 * ldb + j + 1) : pad;
    v.w = (k1 < K && j + 1 < N) ? load_operand<T, MODE>(B + (long long)k1 * ldb + j + 1) : pad;
    reinterpret_cast<float4*>(Bp)[t] = v;
  }
}

// Dense copy of A into an [M][Kp] float panel (row pitch Kp), padding k >= K
// with `pad`.  Used when A's rows are not 16-byte aligned for TMA, or when A
// must be converted (or_and inputs).
template <typename T, int MODE>
__global__ void pack_rows_kernel(const T* __restrict__ A, long long lda, int M, int K, float* __restrict__ Ap,
                                 int Kp, float pad) {
  const long long total = (long long)M * Kp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / Kp);
    const int k = (int)(t - (long long)i * Kp);
    Ap[t] = k < K ? load_operand<T, MODE>(A + (long long)i * lda + k) : pad;
  }
}

// D = id (+) C (or id) for K == 0.
template <typename T>
__global__ void fill_kernel(T* D, long long ldd, int M, int N, T value) {
  const long long total = (long long)M * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / N);
    const int j = (int)(t - (long long)i * N);
    D[(long long)i * ldd + j] = value;
  }
}

// float {-inf,0,1} -> 0/1 of type T (or_and result).
template <typename T>
__global__ void bool_out_kernel(const float* __restrict__ S, long long lds, T* __restrict__ D, long long ldd, int M,
                                int N) {
  const long long total = (long long)M * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / N);
    const int j = (int)(t - (long long)i * N);
    D[(long long)i * ldd + j] = S[(long long)i * lds + j] > 0.5f ? T(1) : T(0);
  }
}

}  // namespace simd2
