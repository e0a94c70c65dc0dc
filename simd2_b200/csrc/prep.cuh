// prep.cuh -- operand preparation kernels (HBM-bound, one pass each).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "common.cuh"

namespace simd2 {

// B'[p][2j+e] = B[2p+e][j] for 2p+e < K and j < N, else `pad`.
// B' has Kp/2 rows of 2*Np floats (Kp, Np are the padded sizes); a float4 of
// B' is (B[2p][j], B[2p+1][j], B[2p][j+1], B[2p+1][j+1]).
template <typename T, int MODE>
__device__ __forceinline__ float load_operand(const T* p) {
  if constexpr (MODE == 1) return (*p != T(0)) ? 1.0f : 0.0f;  // boolean (or_and as max_min on {0,1})
  else return static_cast<float>(*p);
}

// A thread fills 4 columns (two float4 stores); float B with 16-byte aligned
// rows is read with one float4 load per k row where the 4 columns are in range.
template <typename T, int MODE>
__global__ void interleave_pairs_kernel(const T* __restrict__ B, long long ldb, int K, int N,
                                        float* __restrict__ Bp, int Kp, int Np, float pad,
                                        const int* gate = nullptr, const int* gate2 = nullptr) {
  if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
  const long long quads = Np / 4;
  const long long total = (long long)(Kp / 2) * quads;
  constexpr bool kFloat = std::is_same<T, float>::value && MODE == 0;
  const bool vec = kFloat && (ldb % 4 == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / quads);
    const int j = (int)(t - (long long)p * quads) * 4;
    float x[2][4];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int k = 2 * p + r;
      if constexpr (kFloat) {
        if (vec && k < K && j + 4 <= N) {
          const float4 u = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const float*>(B) + (long long)k * ldb + j));
          x[r][0] = u.x, x[r][1] = u.y, x[r][2] = u.z, x[r][3] = u.w;
          continue;
        }
      }
#pragma unroll
      for (int e = 0; e < 4; e++)
        x[r][e] = (k < K && j + e < N) ? load_operand<T, MODE>(B + (long long)k * ldb + j + e) : pad;
    }
    float4* o = reinterpret_cast<float4*>(Bp) + 2 * t;
    o[0] = make_float4(x[0][0], x[1][0], x[0][1], x[1][1]);
    o[1] = make_float4(x[0][2], x[1][2], x[0][3], x[1][3]);
  }
}

// Dense copy of A into an [M][Kp] float panel (row pitch Kp), padding k >= K
// with `pad`.  Used when A's rows are not 16-byte aligned for TMA, or when A
// must be converted (or_and inputs).
template <typename T, int MODE>
__global__ void pack_rows_kernel(const T* __restrict__ A, long long lda, int M, int K, float* __restrict__ Ap,
                                 int Kp, float pad, const int* gate = nullptr, const int* gate2 = nullptr) {
  if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
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

// half -> float (MODE 0) or half -> {0,1} float (MODE 1), [M][K] pitch lda -> dense [M][K].
template <int MODE>
__global__ void half_to_float_kernel(const __half* __restrict__ A, long long lda, int M, int K, float* __restrict__ out) {
  const long long total = (long long)M * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / K);
    const int k = (int)(t - (long long)i * K);
    const float v = __half2float(A[(long long)i * lda + k]);
    out[t] = MODE == 1 ? (v != 0.f ? 1.f : 0.f) : v;
  }
}

// float -> {0,1} float, [M][N] pitch ldc -> dense.
__global__ void float_bool_kernel(const float* __restrict__ C, long long ldc, int M, int N, float* __restrict__ out) {
  const long long total = (long long)M * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / N);
    const int j = (int)(t - (long long)i * N);
    out[t] = C[(long long)i * ldc + j] != 0.f ? 1.f : 0.f;
  }
}

// Change test + copy, the work of comp_update / comp_update2
// (kernel/converge.cuh:6-84): mode 1 |prev-cur| > 1e-4, mode 2 maps cur values
// in (-1,1) to -FLT_MAX first (in cur and prev) then tests inequality, mode 0
// tests bitwise inequality; prev := cur.  One flag word, set by a warp vote.
template <typename T>
__global__ void compare_update_kernel(T* __restrict__ prev, T* __restrict__ cur, long long n, int mode,
                                      int* __restrict__ flag) {
  int ch = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    T c = cur[t];
    const T pv = prev[t];
    if constexpr (std::is_same<T, float>::value) {
      if (mode == 2 && c > T(-1) && c < T(1)) {
        c = T(-3.402823466e+38f);
        cur[t] = c;
      }
      if (mode == 1) ch |= fabsf((float)pv - (float)c) > 0.0001f;
      else ch |= __float_as_uint((float)pv) != __float_as_uint((float)c);
    } else {
      ch |= pv != c;
    }
    prev[t] = c;
  }
  if (__any_sync(0xffffffffu, ch) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// ---------------------------------------------------------------------------
// FP16 selection path (max_min, min_max): path flags and operand packing.
// ---------------------------------------------------------------------------
// flags[0] = 1 (FP16 path), flags[1] = 0 (FP32 path) before the packing.
__global__ void fp16_flags_init_kernel(int* flags) {
  flags[0] = 1;
  flags[1] = 0;
}

__global__ void fp16_flags_finish_kernel(int* flags) { flags[1] = flags[0] ? 0 : 1; }

// The FP16 form of x; *bad is set when the round trip float -> half -> float
// changes x's bits (x is not exactly an FP16 value, NaN included).
__device__ __forceinline__ __half to_half_exact(float x, bool& bad) {
  const __half h = __float2half_rn(x);
  bad |= __float_as_uint(__half2float(h)) != __float_as_uint(x);
  return h;
}

// A [M][K] -> half [M][Kp], NaN padding (k >= K).  Clears flags[0] when an
// entry of A is not exactly an FP16 value.  Kp is a multiple of 8: a thread
// converts 8 consecutive elements of a row and writes them as one 16-byte store.
__global__ void pack_half_rows_kernel(const float* __restrict__ A, long long lda, int M, int K,
                                      __half* __restrict__ out, int Kp, const int* gate, int* flags) {
  if (gate && *gate == 0) return;
  bool bad = false;
  const int groups = Kp >> 3;
  const long long total = (long long)M * groups;
  const bool vec = (lda % 4 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0);
  const __half nanh = __ushort_as_half(0x7e00);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / groups);
    const int k0 = (int)(t - (long long)i * groups) * 8;
    const float* row = A + (long long)i * lda;
    __half h[8];
    if (vec && k0 + 8 <= K) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(row + k0));
      const float4 w = __ldg(reinterpret_cast<const float4*>(row + k0 + 4));
      const float x[8] = {u.x, u.y, u.z, u.w, w.x, w.y, w.z, w.w};
#pragma unroll
      for (int e = 0; e < 8; e++) h[e] = to_half_exact(x[e], bad);
    } else {
#pragma unroll
      for (int e = 0; e < 8; e++) h[e] = k0 + e < K ? to_half_exact(row[k0 + e], bad) : nanh;
    }
    uint32_t wv[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      wv[q] = (uint32_t)__half_as_ushort(h[2 * q]) | ((uint32_t)__half_as_ushort(h[2 * q + 1]) << 16);
    reinterpret_cast<uint4*>(out)[t] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicAnd(flags, 0);
}

// B [K][N] -> k-pair words [Kp/2][Np]: word (p, j) = (half B[2p][j], half B[2p+1][j]),
// NaN padding for k >= K and j >= N.  Clears flags[0] when an entry of B is
// not exactly an FP16 value.  Np is a multiple of 4: a thread forms the words
// of 4 consecutive columns and writes them as one 16-byte store.
__global__ void interleave_half_kernel(const float* __restrict__ B, long long ldb, int K, int N,
                                       __half2* __restrict__ out, int Kp, int Np, const int* gate, int* flags) {
  if (gate && *gate == 0) return;
  bool bad = false;
  const int quads = Np >> 2;
  const long long total = (long long)(Kp / 2) * quads;
  const bool vec = (ldb % 4 == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0);
  const __half nanh = __ushort_as_half(0x7e00);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / quads);
    const int j0 = (int)(t - (long long)p * quads) * 4;
    __half lo[4], hi[4];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int k = 2 * p + r;
      __half* dst = r == 0 ? lo : hi;
      const float* row = B + (long long)k * ldb;
      if (k < K && vec && j0 + 4 <= N) {
        const float4 u = __ldg(reinterpret_cast<const float4*>(row + j0));
        dst[0] = to_half_exact(u.x, bad), dst[1] = to_half_exact(u.y, bad);
        dst[2] = to_half_exact(u.z, bad), dst[3] = to_half_exact(u.w, bad);
      } else {
#pragma unroll
        for (int e = 0; e < 4; e++) dst[e] = (k < K && j0 + e < N) ? to_half_exact(row[j0 + e], bad) : nanh;
      }
    }
    uint32_t wv[4];
#pragma unroll
    for (int e = 0; e < 4; e++)
      wv[e] = (uint32_t)__half_as_ushort(lo[e]) | ((uint32_t)__half_as_ushort(hi[e]) << 16);
    reinterpret_cast<uint4*>(out)[t] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicAnd(flags, 0);
}

// D = (C != 0) as 0/1 of type T.
template <typename T>
__global__ void bool_copy_kernel(const T* __restrict__ C, long long ldc, T* __restrict__ D, long long ldd, int M,
                                 int N) {
  const long long total = (long long)M * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / N);
    const int j = (int)(t - (long long)i * N);
    D[(long long)i * ldd + j] = C[(long long)i * ldc + j] != T(0) ? T(1) : T(0);
  }
}

}  // namespace simd2

namespace simd2 {

// ---------------------------------------------------------------------------
// Operand preparation for the tensor-core paths.  Outputs are K-major with a
// row pitch of Kp elements (Kp a multiple of 8 for BF16, 16 for bytes, so the
// TMA row stride is a multiple of 16 bytes); k in [K, Kp) is zero.
// ---------------------------------------------------------------------------

// x = hi + lo with hi = bf16(x), lo = bf16(x - hi) (both round-to-nearest).
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(__fsub_rn(x, __bfloat162float(hi)));
}

__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// A [M][K] (pitch lda) -> A_hi, A_lo [M][Kp], zeros for k >= K.  Kp is a
// multiple of 8 and hi / lo are 16-byte aligned: a thread converts 8
// consecutive elements of a row (two 16-byte loads when A's rows allow) and
// writes 16 bytes to each output.
__global__ void split_rows_bf16_kernel(const float* __restrict__ A, long long lda, int M, int K,
                                       __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int Kp) {
  const int groups = Kp >> 3;
  const long long total = (long long)M * groups;
  const bool vec = (lda % 4 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / groups);
    const int k0 = (int)(t - (long long)i * groups) * 8;
    const float* row = A + (long long)i * lda;
    float x[8];
    if (vec && k0 + 8 <= K) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(row + k0));
      const float4 w = __ldg(reinterpret_cast<const float4*>(row + k0 + 4));
      x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w, x[4] = w.x, x[5] = w.y, x[6] = w.z, x[7] = w.w;
    } else {
#pragma unroll
      for (int e = 0; e < 8; e++) x[e] = k0 + e < K ? row[k0 + e] : 0.f;
    }
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(x[2 * q], h0, l0);
      split_bf16(x[2 * q + 1], h1, l1);
      hw[q] = pack_bf16x2(h0, h1);
      lw[q] = pack_bf16x2(l0, l1);
    }
    reinterpret_cast<uint4*>(hi)[t] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    reinterpret_cast<uint4*>(lo)[t] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  }
}

// A [M][K] of T -> bytes {0,1} [M][Kp].  Kp is a multiple of 16: a thread
// writes 16 bytes of a row; byte inputs with 16-byte aligned rows are read
// with one 16-byte load and normalised four bytes at a time.
template <typename T>
__global__ void bool_rows_u8_kernel(const T* __restrict__ A, long long lda, int M, int K, uint8_t* __restrict__ out,
                                    int Kp) {
  const int groups = Kp >> 4;
  const long long total = (long long)M * groups;
  constexpr bool kBytes = sizeof(T) == 1;
  const bool vec = kBytes && (lda % 16 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / groups);
    const int k0 = (int)(t - (long long)i * groups) * 16;
    const T* row = A + (long long)i * lda;
    uint32_t w[4];
    if (kBytes && vec && k0 + 16 <= K) {
      const uint4 u = __ldg(reinterpret_cast<const uint4*>(row + k0));
      const uint32_t in[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        // 0x01 in every byte that is nonzero, carry-free
        const uint32_t b = in[q];
        w[q] = bytes_nonzero_01(b);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t v = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int k = k0 + 4 * q + e;
          v |= (uint32_t)(k < K && row[k] != T(0)) << (8 * e);
        }
        w[q] = v;
      }
    }
    reinterpret_cast<uint4*>(out)[t] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// B [K][N] (pitch ldb) -> transposed K-major [N][Kp] through a 32 x 32 shared
// tile (coalesced reads along n, coalesced writes along k).
// MODE 0: BF16 hi/lo split (out0 = hi, out1 = lo); MODE 1: bytes {0,1} (out0).
// colsq (nullable): sum over k of B[k][j]^2 accumulated in FP64 (atomicAdd per
// 32-row tile; the caller zeroes it and rounds it to float afterwards).
template <typename T, int MODE>
__global__ void transpose_prep_kernel(const T* __restrict__ B, long long ldb, int K, int N, void* __restrict__ out0,
                                      void* __restrict__ out1, int Kp, double* __restrict__ colsq = nullptr) {
  __shared__ float tile[32][33];
  const int k0 = blockIdx.y * 32;
  const int j0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int k = k0 + i, j = j0 + threadIdx.x;
    float v = 0.f;
    if (k < K && j < N) {
      const T x = B[(long long)k * ldb + j];
      if constexpr (MODE == 1) v = (x != T(0)) ? 1.f : 0.f;
      else v = static_cast<float>(x);
    }
    tile[i][threadIdx.x] = v;
  }
  __syncthreads();
  if (colsq != nullptr && threadIdx.y == 0 && j0 + (int)threadIdx.x < N) {
    double s = 0.0;
    for (int i = 0; i < 32; i++) {
      const double v = tile[i][threadIdx.x];
      s += v * v;
    }
    atomicAdd(colsq + j0 + threadIdx.x, s);
  }
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int j = j0 + i, k = k0 + threadIdx.x;
    if (j < N && k < Kp) {
      const float v = tile[threadIdx.x][i];
      const long long o = (long long)j * Kp + k;
      if constexpr (MODE == 1) {
        static_cast<uint8_t*>(out0)[o] = (uint8_t)(v != 0.f);
      } else {
        __nv_bfloat16 h, l;
        split_bf16(v, h, l);
        static_cast<__nv_bfloat16*>(out0)[o] = h;
        static_cast<__nv_bfloat16*>(out1)[o] = l;
      }
    }
  }
}

// or_and's B operand for bytes: B [K][N] (pitch ldb) -> out [N][Kp], 1 where
// B is nonzero, zeros for K <= k < Kp (transpose_prep_kernel<T, 1>'s result).
// One 64 x 64 tile per block of 256 threads: a thread reads 16 bytes of a row
// of B (one 16-byte load where B allows) and writes 16 bytes of a row of out;
// the shared tile's 68-byte rows keep both phases at most 2-way bank
// conflicted.  Kp is a multiple of 16, out 16-byte aligned; the grid covers
// ceil(N / 64) x ceil(Kp / 64) tiles.
__global__ void __launch_bounds__(256) transpose_bool_u8_kernel(const uint8_t* __restrict__ B, long long ldb, int K,
                                                                int N, uint8_t* __restrict__ out, int Kp) {
  __shared__ uint32_t tile[64][17];
  const int t = threadIdx.x;
  const int k0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
  {
    const int r = t >> 2, c0 = (t & 3) * 16;
    const int k = k0 + r, j = j0 + c0;
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if (k < K && j < N) {
      const uint8_t* src = B + (long long)k * ldb + j;
      if (j + 16 <= N && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src));
        w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
      } else {
        for (int e = 0; e < 16 && j + e < N; e++) w[e >> 2] |= (uint32_t)src[e] << (8 * (e & 3));
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) tile[r][(c0 >> 2) + q] = bytes_nonzero_01(w[q]);
  }
  __syncthreads();
  const int jj = t >> 2, kc = (t & 3) * 16;
  const int jo = j0 + jj, ko = k0 + kc;
  if (jo < N && ko < Kp) {
    const int sh = 8 * (jj & 3);
    uint32_t o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint32_t x = 0u;
#pragma unroll
      for (int b = 0; b < 4; b++) x |= ((tile[kc + 4 * q + b][jj >> 2] >> sh) & 0xffu) << (8 * b);
      o[q] = x;
    }
    *reinterpret_cast<uint4*>(out + (long long)jo * Kp + ko) = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// Squared row norms of A [M][K], accumulated in FP64, rounded to float.
__global__ void row_norms_kernel(const float* __restrict__ A, long long lda, int M, int K, float* __restrict__ out) {
  const int warps = blockDim.x / 32;
  for (int i = blockIdx.x * warps + threadIdx.x / 32; i < M; i += gridDim.x * warps) {
    double s = 0.0;
    for (int k = threadIdx.x % 32; k < K; k += 32) {
      const double v = A[(long long)i * lda + k];
      s += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x % 32 == 0) out[i] = (float)s;
  }
}

// double -> float (norms accumulated in FP64).
__global__ void round_norms_kernel(const double* __restrict__ in, int n, float* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) out[j] = (float)in[j];
}

}  // namespace simd2
