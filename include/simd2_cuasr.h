/*
 * simd2_cuasr.h -- exact-signature drop-ins for escalab/SIMD2 callers.
 *
 * Replaces, for existing callers, the declarations of
 *   kernel/srgemm.cuh        cuasr_<op>_srsgemm x9 (lines 28, 89, 147, 213, 269,
 *                            326, 384, 442, 552): column-major cuASR srgemm
 *   kernel/tensor_srgemm.cuh enum op (18-26), tensor_srgemm (197-218)
 *   kernel/converge.cuh      comp_update / comp_update2 (16-84)
 *   apps/pld/cuASR/knncuda.h knn_mxu (65-73), the PLD k-NN entry
 * with inline shims over the libsimd2 C ABI (simd2.h).  Include this header
 * instead of those three and link libsimd2; no cuASR / CUTLASS needed.
 *
 * Column-major D(M x N) = A(M x K) (x) B(K x N) (+) C with leading dimensions
 * lda, ldb, ldc (D uses ldc, as in cuASR) is the row-major problem on the
 * transposes D^T = B^T (x) A^T (+) C^T; every (x) here is commutative, so the
 * shim swaps the operands and the sizes and calls simd2_srgemm.
 */
#ifndef SIMD2_CUASR_H
#define SIMD2_CUASR_H

#include <cuda_fp16.h>
#include <stdlib.h>

#include "simd2.h"

#define SIMD2_CUASR_FLOAT_SHIM(NAME, OP)                                                            \
  inline int NAME(int M, int N, int K, float const* A, int lda, float const* B, int ldb, float* C,  \
                  int ldc, float* D, bool do_epilogue, cudaStream_t stream = nullptr) {              \
    return simd2_srgemm(OP, N, M, K, B, ldb, A, lda, C, ldc, D, ldc, do_epilogue ? 1 : 0, stream); \
  }

SIMD2_CUASR_FLOAT_SHIM(cuasr_minplus_srsgemm, SIMD2_MIN_PLUS)
SIMD2_CUASR_FLOAT_SHIM(cuasr_plusmul_srsgemm, SIMD2_PLUS_MUL)
SIMD2_CUASR_FLOAT_SHIM(cuasr_maxplus_srsgemm, SIMD2_MAX_PLUS)
SIMD2_CUASR_FLOAT_SHIM(cuasr_maxmin_srsgemm, SIMD2_MAX_MIN)
SIMD2_CUASR_FLOAT_SHIM(cuasr_maxmul_srsgemm, SIMD2_MAX_MUL)
SIMD2_CUASR_FLOAT_SHIM(cuasr_minmul_srsgemm, SIMD2_MIN_MUL)
SIMD2_CUASR_FLOAT_SHIM(cuasr_minmax_srsgemm, SIMD2_MIN_MAX)
/* (sic) the reference spells this one "plusmiussquare" */
SIMD2_CUASR_FLOAT_SHIM(cuasr_plusmiussquare_srsgemm, SIMD2_MINUS_SQUARE)

inline int cuasr_orand_srsgemm(int M, int N, int K, int const* A, int lda, int const* B, int ldb, int* C,
                               int ldc, int* D, bool do_epilogue, cudaStream_t stream = nullptr) {
  return simd2_srgemm_orand_i32(N, M, K, B, ldb, A, lda, C, ldc, D, ldc, do_epilogue ? 1 : 0, stream);
}

#undef SIMD2_CUASR_FLOAT_SHIM

/* kernel/tensor_srgemm.cuh:18-26 */
enum op { min_plus, plus_mul, max_plus, max_min, max_mul, min_mul, min_max, or_and, minus_square };

/* kernel/tensor_srgemm.cuh:197-218: row-major, FP16 A/B, FP32 C/D, default
 * stream, asynchronous; -1 unless m, n, k are multiples of 16. */
extern "C" inline int tensor_srgemm(half* a, half* b, float* c, float* d, int m, int n, int k, bool do_epilogue,
                                    enum op opcode) {
  if (m % 16 != 0 || n % 16 != 0 || k % 16 != 0) return -1;
  return simd2_srgemm_f16((simd2_op)opcode, m, n, k, a, k, b, n, c, n, d, n, do_epilogue ? 1 : 0, nullptr) == 0
             ? 0
             : -1;
}

/* kernel/converge.cuh:16-30: |prev-cur| > 1e-4 test, copies cur into prev,
 * synchronous.  `check` (device) is not needed; check_h[0] gets the flag. */
inline bool comp_update(float* prev, float* cur, int* check, int* check_h, int M, int N) {
  (void)check;
  int ch = 0;
  simd2_compare_update(prev, cur, M, N, SIMD2_CONV_TOL, &ch, nullptr);
  if (check_h) check_h[0] = ch;
  return ch != 0;
}

/* kernel/converge.cuh:45-58: APLP variant (cur values in (-1,1) -> -FLT_MAX). */
inline bool comp_update2(float* prev, float* cur, int* check, int* check_h, int M, int N) {
  (void)check;
  int ch = 0;
  simd2_compare_update(prev, cur, M, N, SIMD2_CONV_APLP, &ch, nullptr);
  if (check_h) check_h[0] = ch;
  return ch != 0;
}

/* kernel/converge.cuh:71-84: int version (exact inequality). */
inline bool comp_update(int* prev, int* cur, int* check, int* check_h, int M, int N) {
  (void)check;
  int ch = 0;
  simd2_compare_update_i32(prev, cur, M, N, &ch, nullptr);
  if (check_h) check_h[0] = ch;
  return ch != 0;
}

/* apps/pld/cuASR/knncuda.h:65-73, knn_mxu: the k nearest references of
 * every query.  Host arrays in the reference's layouts: ref [ref_nb][dim]
 * (the caller's transposed copy, apps/pld/cuASR/test.cpp:56-65), query
 * [dim][query_nb], knn_dist / knn_index [k][query_nb] (distances ascending,
 * 0-based reference indices, ties to the lower index).  *kernel_time grows by
 * the seconds spent in simd2_knn, as the reference adds its srgemm time.
 * Allocates and frees its device buffers per call, as the reference does. */
inline bool knn_mxu(const float* ref, int ref_nb, const float* query, int query_nb, int dim, int k, float* knn_dist,
                    int* knn_index, double* kernel_time) {
  if (ref_nb < 1 || query_nb < 1 || dim < 1 || k < 1 || k > ref_nb) return false;
  const size_t qd = (size_t)query_nb * dim, rd = (size_t)ref_nb * dim, qk = (size_t)query_nb * k;
  float* hq = (float*)malloc(qd * sizeof(float));
  float* hd = (float*)malloc(qk * sizeof(float));
  int* hi = (int*)malloc(qk * sizeof(int));
  float *dq = nullptr, *dr = nullptr, *dd = nullptr;
  int* di = nullptr;
  bool ok = hq && hd && hi && cudaMalloc((void**)&dq, qd * sizeof(float)) == cudaSuccess &&
            cudaMalloc((void**)&dr, rd * sizeof(float)) == cudaSuccess &&
            cudaMalloc((void**)&dd, qk * sizeof(float)) == cudaSuccess &&
            cudaMalloc((void**)&di, qk * sizeof(int)) == cudaSuccess;
  if (ok) {
    for (int q = 0; q < query_nb; q++)  // [dim][query_nb] -> [query_nb][dim]
      for (int d = 0; d < dim; d++) hq[(size_t)q * dim + d] = query[(size_t)d * query_nb + q];
    ok = cudaMemcpy(dq, hq, qd * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(dr, ref, rd * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  if (ok) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, nullptr);
    ok = simd2_knn(dq, query_nb, dim, dr, ref_nb, dim, dim, k, dd, di, k, nullptr) == 0;
    cudaEventRecord(e1, nullptr);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (kernel_time) *kernel_time += ms / 1e3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (ok)
    ok = cudaMemcpy(hd, dd, qk * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(hi, di, qk * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ok)
    for (int q = 0; q < query_nb; q++)  // [query_nb][k] -> [k][query_nb]
      for (int j = 0; j < k; j++) {
        knn_dist[(size_t)j * query_nb + q] = hd[(size_t)q * k + j];
        knn_index[(size_t)j * query_nb + q] = hi[(size_t)q * k + j];
      }
  cudaFree(dq);
  cudaFree(dr);
  cudaFree(dd);
  cudaFree(di);
  free(hq);
  free(hd);
  free(hi);
  return ok;
}

#endif /* SIMD2_CUASR_H */
