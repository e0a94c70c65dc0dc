// ref_host_srgemm.cpp -- thin C wrapper around the reference's own
// mmo::host_srgemm (escalab/SIMD2 kernel/host_srgemm.h:17-85), compiled from
// the header where it lies in the reference tree (see oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: used to pin the C restatement (simd2_oracle.c)
// and as the CPU baseline ("kind": "reference") in bench.py.  Rows are split
// into panels across std::threads; each thread calls the unchanged reference
// function on its own rows (M = panel rows, A and D offset to the panel).
#include <cstdint>
#include <thread>
#include <vector>
#include "host_srgemm.h"

namespace {
using fop = float (*)(float, float);
using iop = int (*)(int, int);

bool pick(int op, fop* add, fop* mul) {
  switch (op) {
    case 0: *add = mmo::minimum<float>; *mul = mmo::plus<float>; return true;        // min_plus
    case 1: *add = mmo::plus<float>; *mul = mmo::multiplies<float>; return true;     // plus_mul
    case 2: *add = mmo::maximum<float>; *mul = mmo::plus<float>; return true;        // max_plus
    case 3: *add = mmo::maximum<float>; *mul = mmo::minimum<float>; return true;     // max_min
    case 4: *add = mmo::maximum<float>; *mul = mmo::multiplies<float>; return true;  // max_mul
    case 5: *add = mmo::minimum<float>; *mul = mmo::multiplies<float>; return true;  // min_mul
    case 6: *add = mmo::minimum<float>; *mul = mmo::maximum<float>; return true;     // min_max
    case 8: *add = mmo::plus<float>; *mul = mmo::minussquare<float>; return true;    // minus_square
    default: return false;
  }
}

template <typename T, typename F>
void panels(int M, int nthreads, F&& body) {
  if (M <= 0) return;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > M) nthreads = M;
  std::vector<std::thread> th;
  for (int t = 1; t < nthreads; t++)
    th.emplace_back(body, (int)((int64_t)M * t / nthreads), (int)((int64_t)M * (t + 1) / nthreads));
  body(0, (int)((int64_t)M / nthreads));
  for (auto& x : th) x.join();
}
}  // namespace

extern "C" int ref_srgemm_f32(int op, int M, int N, int K, const float* A, const float* B, const float* C,
                              float* D, int do_epilogue, int nthreads) {
  fop add, mul;
  if (!pick(op, &add, &mul)) return -1;
  panels<float>(M, nthreads, [&](int r0, int r1) {
    if (r1 <= r0) return;
    mmo::host_srgemm<float>(r1 - r0, N, K, const_cast<float*>(A) + (size_t)r0 * K, K, const_cast<float*>(B), N,
                            const_cast<float*>(C) + (size_t)r0 * N, N, D + (size_t)r0 * N, do_epilogue != 0,
                            add, mul);
  });
  return 0;
}

extern "C" int ref_srgemm_i32_orand(int M, int N, int K, const int32_t* A, const int32_t* B, const int32_t* C,
                                    int32_t* D, int do_epilogue, int nthreads) {
  panels<int>(M, nthreads, [&](int r0, int r1) {
    if (r1 <= r0) return;
    mmo::host_srgemm<int>(r1 - r0, N, K, const_cast<int32_t*>(A) + (size_t)r0 * K, K, const_cast<int32_t*>(B), N,
                          const_cast<int32_t*>(C) + (size_t)r0 * N, N, D + (size_t)r0 * N, do_epilogue != 0,
                          (iop)mmo::bin_or<int>, (iop)mmo::bin_and<int>);
  });
  return 0;
}
