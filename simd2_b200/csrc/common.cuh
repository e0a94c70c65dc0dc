// common.cuh -- shared device helpers for libsimd2 (sm_100a only).
//
// mbarrier / TMA wrappers are written as inline PTX; every wait is bounded by
// wall time (%globaltimer) so that a lost arrival turns into an error word the
// host can read instead of a hung GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/simd2.h"

namespace simd2 {

// Device-side error word (SIMD2_ERR_TIMEOUT etc.), read by simd2_device_status().
// The library is one translation unit (capi.cu includes every kernel header),
// so this is the single definition.
__device__ int g_device_status = 0;
// Largest wait-site id that timed out (0 = none); sites are numbered per kernel.
__device__ int g_timeout_site = 0;

// Wall-time limit of one bounded wait, in nanoseconds (2 s).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on phase `parity`.  Returns false if kWaitLimitNs elapsed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    for (int i = 0; i < 64; i++)
      if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// 2D tiled TMA load (no multicast) into this CTA's shared memory; completion
// is signalled as transaction bytes on `bar`.  x is the innermost coordinate.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

__device__ __forceinline__ void report_error(int code) { atomicOr(&g_device_status, code); }
__device__ __forceinline__ void report_timeout(int site) {
  atomicOr(&g_device_status, SIMD2_ERR_TIMEOUT);
  atomicMax(&g_timeout_site, site);
}

// Self-test of the bounded wait: waits on a fresh barrier that nothing
// arrives on (its phase never completes) for at most limit_ns, then reports
// SIMD2_ERR_TIMEOUT with wait-site 99 through the normal error word and
// returns.  Nothing faults or hangs: the wait simply runs out.
__global__ void wait_timeout_selftest_kernel(uint64_t limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, limit_ns)) report_timeout(99);
}


// ---------------------------------------------------------------------------
// Semiring operators.  The add step keeps host_srgemm's accumulator-first
// form: std::min(D,p) == (p < D ? p : D) and std::max(D,p) == (D < p ? p : D)
// agree with PTX min/max whenever neither operand is NaN or a signed zero; a
// NaN product is dropped by both (the accumulator is never NaN).
// Three-operand min/max (PTX ISA 8.8, .f32 with three sources, sm_100+) folds
// two products into the accumulator in one instruction; min/max is
// associative and commutative on non-NaN values, so this is bit-exact.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min2f(float a, float b) {
  float r;
  asm("min.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float max2f(float a, float b) {
  float r;
  asm("max.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

template <int OP>
struct Semiring;

// (+) = min
struct MinAdd {
  static constexpr bool kSum = false;
  __device__ static float identity() { return __int_as_float(0x7f800000); }
  __device__ static float add(float acc, float p) { return min2f(acc, p); }
  __device__ static float add3(float acc, float p, float q) { return min3f(acc, p, q); }
};
// (+) = max
struct MaxAdd {
  static constexpr bool kSum = false;
  __device__ static float identity() { return __int_as_float(0xff800000); }
  __device__ static float add(float acc, float p) { return max2f(acc, p); }
  __device__ static float add3(float acc, float p, float q) { return max3f(acc, p, q); }
};

template <>
struct Semiring<SIMD2_MIN_PLUS> : MinAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return __fadd2_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
};
template <>
struct Semiring<SIMD2_MAX_PLUS> : MaxAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return __fadd2_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
};
template <>
struct Semiring<SIMD2_MIN_MUL> : MinAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
};
template <>
struct Semiring<SIMD2_MAX_MUL> : MaxAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
};
// max_min: (x) = min
template <>
struct Semiring<SIMD2_MAX_MIN> : MaxAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return make_float2(min2f(a.x, b.x), min2f(a.y, b.y)); }
  __device__ static float mul(float a, float b) { return min2f(a, b); }
};
// min_max: (x) = max
template <>
struct Semiring<SIMD2_MIN_MAX> : MinAdd {
  __device__ static float2 mul2(float2 a, float2 b) { return make_float2(max2f(a.x, b.x), max2f(a.y, b.y)); }
  __device__ static float mul(float a, float b) { return max2f(a, b); }
};

// Per byte of x: 1 where the byte is nonzero, else 0 (no carry crosses a byte:
// (b & 0x7f) + 0x7f <= 0xfe, and its top bit is set iff b & 0x7f != 0).
__device__ __forceinline__ uint32_t bytes_nonzero_01(uint32_t x) {
  return ((((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x) & 0x80808080u) >> 7;
}

}  // namespace simd2
