// spgemm.cuh -- semiring SpGEMM on CSR matrices, for inputs too sparse for
// the dense kernels (the regime of density_verification/sp_gemm_comp.cu,
// which times cuSPARSE SpGEMM against dense GEMM as the density falls).
//
// D = A (x) B [(+) C] where an absent entry is the semiring's add identity.
// That is exact only where the add identity annihilates the multiply on the
// stored values: min_plus (+inf), max_plus (-inf), max_min (-inf), min_max
// (+inf), plus_mul (0).  The result stores every column reached through a
// stored A[i][k] and B[k][j] (or stored in C), in increasing column order.
//
// Row-wise (Gustavson) accumulation.  Persistent CTAs take rows from an
// atomic counter; a CTA keeps, for its current row, a bitmap of touched
// columns in shared memory and the running values next to it in shared
// memory (N <= 16384) or in its own slice of a global scratch array.
// For plus_mul the row's A entries are visited in increasing k; for each k
// the threads spread over B's row k (distinct columns, so no two threads meet
// on one column) and a barrier separates consecutive k.  Every output
// therefore receives its products in increasing k -- the host_srgemm order
// (kernel/host_srgemm.h:17-49) -- starting from the add identity, then the C
// term: bit-identical to the dense contract.  The min/max adds are
// order-independent on non-NaN values, so for them each warp takes its own
// A entries and folds products with atomic min / max on order-preserving
// keys: the same bits without a barrier per k.  The bitmap is scanned in word
// order to write the row's columns sorted.
//
// Two passes share the kernel: COUNT writes the row's nonzero count (no
// values, no barriers per k), FILL writes columns and values at the offsets
// the host formed from the counts -- or, with DENSE, the values straight into
// a dense matrix prefilled with the identity (no offsets needed).
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kSpThreads = 512;

template <int OP>
struct SpOps;
template <>
struct SpOps<SIMD2_MIN_PLUS> {
  __device__ static float ident() { return __int_as_float(0x7f800000); }
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
  __device__ static float add(float d, float p) { return (p < d) ? p : d; }
};
template <>
struct SpOps<SIMD2_MAX_PLUS> {
  __device__ static float ident() { return __int_as_float(0xff800000); }
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
  __device__ static float add(float d, float p) { return (d < p) ? p : d; }
};
template <>
struct SpOps<SIMD2_MAX_MIN> {
  __device__ static float ident() { return __int_as_float(0xff800000); }
  __device__ static float mul(float a, float b) { return (b < a) ? b : a; }
  __device__ static float add(float d, float p) { return (d < p) ? p : d; }
};
template <>
struct SpOps<SIMD2_MIN_MAX> {
  __device__ static float ident() { return __int_as_float(0x7f800000); }
  __device__ static float mul(float a, float b) { return (a < b) ? b : a; }
  __device__ static float add(float d, float p) { return (p < d) ? p : d; }
};
template <>
struct SpOps<SIMD2_PLUS_MUL> {
  __device__ static float ident() { return 0.f; }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ static float add(float d, float p) { return __fadd_rn(d, p); }
};

struct SpArgs {
  int M, N, K;
  int a_nnz, b_nnz, c_nnz;  // entries in the column / value arrays (reads are clamped to them)
  long long d_cap;          // FILL: entries in dj / dv (writes are clamped to them)
  const int* ap;  // A: M + 1 offsets, columns (the k of B's rows), values
  const int* aj;
  const float* av;
  const int* bp;  // B: K + 1 offsets, columns < N, values
  const int* bj;
  const float* bv;
  const int* cp;  // optional C (epilogue), M + 1 offsets; null when absent
  const int* cj;
  const float* cv;
  const int* dp;  // FILL: output offsets (M + 1)
  int* dj;        // FILL: output columns
  float* dv;      // FILL: output values
  float* dense;   // FILL into a dense matrix (DENSE): D rows of pitch ldd, prefilled with the identity
  uint8_t* dense_u8;  // or, for a Boolean closure, a 0/1 byte matrix prefilled with 0 (touched -> 1)
  long long ldd;
  int* row_nnz;   // COUNT: per-row nonzero count
  float* acc;     // gridDim.x * N floats of scratch (FILL)
  int* next_row;  // atomic row counter, zero before the launch
};

// Exclusive prefix sum of x over the block (kSpThreads threads); total in *total.
__device__ __forceinline__ int block_exclusive_scan(int x, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  int base = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kSpThreads / 32; w++) {
    const int t = s_warp[w];
    if (w < warp) base += t;
    tot += t;
  }
  __syncthreads();
  *total = tot;
  return base + v - x;
}

// min/max adds fold in any order on non-NaN values, so their FILL runs
// without the per-k barrier: values live in the scratch as order-preserving
// unsigned keys (larger float, larger key) folded with atomicMin / atomicMax.
// -0.0 is the one value whose key differs from an equal float's; operands
// hold none (the precondition), and a sum of two values that are not -0.0,
// or the selection of one of them, is never -0.0.
// kUntouched lies past every float's key on the side the fold moves away
// from (all ones for min, zero for max), so a key still at kUntouched marks a
// column no product reached.
template <int OP>
struct SpKey {
  static constexpr bool kUnordered = OP != SIMD2_PLUS_MUL;
  static constexpr bool kMin = OP == SIMD2_MIN_PLUS || OP == SIMD2_MIN_MAX;
  static constexpr uint32_t kUntouched = kMin ? 0xffffffffu : 0u;
  __device__ static uint32_t key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  }
  __device__ static float value(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }
  // A NaN product is dropped, as the dense min / max drops it; it still
  // reaches its column, so the add identity is folded in its place.
  __device__ static void fold(uint32_t* p, float v, float ident) {
    const uint32_t k = key(v != v ? ident : v);
    if constexpr (kMin) atomicMin(p, k);
    else atomicMax(p, k);
  }
};

// Words of the column bitmap, rounded up so that an accumulator array placed
// after it in shared memory starts 16-byte aligned.
__host__ __device__ constexpr int sp_bitmap_words(int n) { return ((n + 31) / 32 + 3) & ~3; }

// Bytes of shared memory for the COUNT pass's column flags (one byte per
// column, rounded to 16 bytes for the vector clears).
__host__ __device__ constexpr int sp_flag_bytes(int n) { return (n + 15) & ~15; }
// Shared-memory accumulators: N rounded up to 4, so that the keys-only
// write-out reads them 4 at a time (the padding stays untouched).
__host__ __device__ constexpr int sp_acc_words(int n) { return (n + 3) & ~3; }

// SMEM (N <= 16384): the row's state lives in shared memory --
//   COUNT: one flag byte per column, set with plain stores (every writer
//     stores 1, so no atomics: the lanes of a warp that reach neighbouring
//     columns of a near-dense B row would serialise on one bitmap word);
//   FILL, min/max adds: the accumulator keys alone (a key at kUntouched is a
//     column no product reached; no bitmap, no atomicOr per product);
//   FILL, plus_mul: the bitmap and the N accumulators after it.
// Otherwise the bitmap sits in shared memory and the accumulators in the
// CTA's slice of the global scratch.
//
// KEYS = false keeps the bitmap in the min/max FILL too (marking it costs an
// atomicOr per product, the write-out walks N/32 words instead of N keys):
// the host picks it for results sparser than 1/32 on average.
template <int OP, bool COUNT, bool DENSE = false, bool SMEM = false, bool KEYS = true>
__global__ void __launch_bounds__(kSpThreads, 2048 / kSpThreads) spgemm_rows_kernel(SpArgs a) {
  using O = SpOps<OP>;
  using KY = SpKey<OP>;
  // warp-parallel over k: COUNT always, FILL for the order-independent adds
  constexpr bool kWarpK = COUNT || KY::kUnordered;
  constexpr bool kBytes = SMEM && COUNT;                      // flag bytes
  constexpr bool kKeysOnly = KEYS && SMEM && !COUNT && KY::kUnordered;  // keys, no bitmap
  constexpr uint32_t kUntouched = KY::kUntouched;
  extern __shared__ __align__(16) uint32_t sp_smem[];
  uint32_t* bitmap = sp_smem;  // ceil(N / 32) words
  uint8_t* flags = reinterpret_cast<uint8_t*>(sp_smem);
  __shared__ int s_row;
  __shared__ int s_warp[kSpThreads / 32];
  const int words = (a.N + 31) >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* acc = SMEM ? reinterpret_cast<float*>(sp_smem + sp_bitmap_words(a.N)) : a.acc + (size_t)blockIdx.x * a.N;
  uint32_t* acck = reinterpret_cast<uint32_t*>(acc);
  const float ident = O::ident();
  if constexpr (!COUNT && KY::kUnordered) {
    // the accumulators start untouched (keys only) or at the identity; every
    // row puts back what it touched
    const uint32_t ik = kKeysOnly ? kUntouched : KY::key(ident);
    const int n_acc = kKeysOnly ? sp_acc_words(a.N) : a.N;
    for (int j = threadIdx.x; j < n_acc; j += kSpThreads) acck[j] = ik;
  }
  // the value of touched column j once the row's folds are done
  auto result = [&](int j) -> float {
    if constexpr (KY::kUnordered) {
      if constexpr (SMEM) {
        const float v = KY::value(acck[j]);
        acck[j] = KY::key(ident);
        return v;
      } else {
        const float v = KY::value(__ldcg(acck + j));
        __stcg(acck + j, KY::key(ident));
        return v;
      }
    } else {
      return acc[j];
    }
  };
  while (true) {
    if (threadIdx.x == 0) s_row = atomicAdd(a.next_row, 1);
    if constexpr (kBytes) {
      for (int w = threadIdx.x; w < sp_flag_bytes(a.N) / 16; w += kSpThreads)
        reinterpret_cast<uint4*>(flags)[w] = make_uint4(0u, 0u, 0u, 0u);
    } else if constexpr (!kKeysOnly) {
      for (int w = threadIdx.x; w < words; w += kSpThreads) bitmap[w] = 0u;
    }
    __syncthreads();
    const int r = s_row;
    if (r >= a.M) break;
    // Offsets and indices are validated by the host pass before any launch;
    // the clamps keep every access inside the arrays whatever they hold.
    const int e1 = min(a.ap[r + 1], a.a_nnz);
    if constexpr (kWarpK) {
      // One warp per A entry (k), its lanes over B's row k; no order between k.
      // The loads form a chain (A's column k, then B's row offsets, then B's
      // columns and values), so the next entry's k and offsets are fetched
      // before the current B row is walked, and the walk keeps four loads of
      // B's columns (and values) in flight per lane.
      constexpr int kStride = kSpThreads / 32;
      int e = max(a.ap[r], 0) + warp;
      int kn = -1, f0n = 0, f1n = 0;
      float avn = 0.f;
      auto fetch = [&](int ee) {
        kn = -1;
        if (ee < e1) {
          const int k = a.aj[ee];
          if ((unsigned)k < (unsigned)a.K) {  // uniform across the warp
            kn = k;
            f0n = max(a.bp[k], 0);
            f1n = min(a.bp[k + 1], a.b_nnz);
            if constexpr (!COUNT) avn = a.av[ee];
          }
        }
      };
      fetch(e);
      for (; e < e1; e += kStride) {
        const int k = kn, f0 = f0n, f1 = f1n;
        const float av = avn;
        fetch(e + kStride);
        if (k < 0) continue;
        auto put = [&](int j, float bvv) {
          if ((unsigned)j >= (unsigned)a.N) return;
          if constexpr (kBytes) flags[j] = 1;
          else if constexpr (!kKeysOnly) atomicOr(&bitmap[j >> 5], 1u << (j & 31));
          if constexpr (!COUNT) KY::fold(acck + j, O::mul(av, bvv), ident);
        };
        // four predicated loads per lane per round trip, so a row under 128
        // entries costs one round trip too
        for (int f = f0 + lane; f < f1; f += 128) {
          int j[4];
          float bvv[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int ff = f + 32 * u;
            j[u] = ff < f1 ? a.bj[ff] : -1;
            bvv[u] = (COUNT || ff >= f1) ? 0.f : a.bv[ff];
          }
#pragma unroll
          for (int u = 0; u < 4; u++) put(j[u], bvv[u]);
        }
      }
    } else {
      for (int e = max(a.ap[r], 0); e < e1; e++) {
        const int k = a.aj[e];
        if ((unsigned)k >= (unsigned)a.K) continue;  // uniform across the block
        const float av = a.av[e];
        const int f1 = min(a.bp[k + 1], a.b_nnz);
        for (int f = max(a.bp[k], 0) + threadIdx.x; f < f1; f += kSpThreads) {
          const int j = a.bj[f];
          if ((unsigned)j >= (unsigned)a.N) continue;
          const uint32_t bit = 1u << (j & 31);
          const uint32_t old = atomicOr(&bitmap[j >> 5], bit);
          acc[j] = O::add((old & bit) ? acc[j] : ident, O::mul(av, a.bv[f]));
        }
        __syncthreads();  // the next k sees this k's values, in order
      }
    }
    if (a.cp) {
      // epilogue: D = D (+) C over C's stored entries (after all products in
      // the ordered fill, the host_srgemm order)
      const int g1 = min(a.cp[r + 1], a.c_nnz);
      for (int f = max(a.cp[r], 0) + threadIdx.x; f < g1; f += kSpThreads) {
        const int j = a.cj[f];
        if ((unsigned)j >= (unsigned)a.N) continue;
        if constexpr (kBytes) {
          flags[j] = 1;
        } else if constexpr (kKeysOnly) {
          KY::fold(acck + j, a.cv[f], ident);
        } else {
          const uint32_t bit = 1u << (j & 31);
          const uint32_t old = atomicOr(&bitmap[j >> 5], bit);
          if constexpr (!COUNT) {
            if constexpr (KY::kUnordered) KY::fold(acck + j, a.cv[f], ident);
            else acc[j] = O::add((old & bit) ? acc[j] : ident, a.cv[f]);
          }
        }
      }
    }
    __syncthreads();
    if constexpr (kBytes) {
      // flag bytes are 0 or 1, so a word's popcount is its flag count
      int cnt = 0;
      for (int w = threadIdx.x; w < sp_flag_bytes(a.N) / 16; w += kSpThreads) {
        const uint4 f = reinterpret_cast<const uint4*>(flags)[w];
        cnt += __popc(f.x) + __popc(f.y) + __popc(f.z) + __popc(f.w);
      }
      int total;
      block_exclusive_scan(cnt, s_warp, &total);
      if (threadIdx.x == 0) a.row_nnz[r] = total;
    } else if constexpr (kKeysOnly && DENSE) {
      // the touched columns straight into the dense row (the rest holds the identity)
      float* drow = a.dense_u8 ? nullptr : a.dense + (long long)r * a.ldd;
      uint8_t* brow = a.dense_u8 ? a.dense_u8 + (long long)r * a.ldd : nullptr;
      // four keys per thread and load (the padding past N is untouched)
      for (int j = 4 * threadIdx.x; j < a.N; j += 4 * kSpThreads) {
        const uint4 k4 = *reinterpret_cast<const uint4*>(acck + j);
        const uint32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
        for (int s = 0; s < 4; s++) {
          if (kk[s] != kUntouched) {
            acck[j + s] = kUntouched;
            if (brow) brow[j + s] = 1;
            else drow[j + s] = KY::value(kk[s]);
          }
        }
      }
    } else if constexpr (kKeysOnly) {
      // columns in increasing order: warp w owns the contiguous column range
      // [w * span, (w + 1) * span) (span a multiple of 128), lane l the keys
      // 4l..4l+3 of each 128-column step, read with one 16-byte load.  A first
      // pass counts the range, a second writes it at the row offset plus the
      // counts of the warps before it, skipping steps with nothing touched.
      constexpr int kWarps = kSpThreads / 32;
      const int span = ((a.N + kWarps * 128 - 1) / (kWarps * 128)) * 128;
      const int c0 = warp * span, c1 = min(a.N, c0 + span);
      int cnt = 0;
      for (int jb = c0; jb < c1; jb += 128) {
        const int j = jb + 4 * lane;
        if (j < c1) {
          const uint4 k4 = *reinterpret_cast<const uint4*>(acck + j);
          cnt += (k4.x != kUntouched) + (k4.y != kUntouched) + (k4.z != kUntouched) + (k4.w != kUntouched);
        }
      }
      cnt = __reduce_add_sync(0xffffffffu, cnt);
      if (lane == 0) s_warp[warp] = cnt;
      __syncthreads();
      long long pos = a.dp[r];
      for (int w = 0; w < warp; w++) pos += s_warp[w];
      const long long out_end = min((long long)a.dp[r + 1], a.d_cap);
      for (int jb = c0; jb < c1; jb += 128) {
        const int j = jb + 4 * lane;
        uint4 k4 = make_uint4(kUntouched, kUntouched, kUntouched, kUntouched);
        if (j < c1) k4 = *reinterpret_cast<const uint4*>(acck + j);
        const uint32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
        const int c = (kk[0] != kUntouched) + (kk[1] != kUntouched) + (kk[2] != kUntouched) + (kk[3] != kUntouched);
        if (!__any_sync(0xffffffffu, c != 0)) continue;  // uniform across the warp
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        long long at = pos + incl - c;
#pragma unroll
        for (int s = 0; s < 4; s++) {
          if (kk[s] != kUntouched) {
            acck[j + s] = kUntouched;
            if (at >= 0 && at < out_end) {
              a.dj[at] = j + s;
              a.dv[at] = KY::value(kk[s]);
            }
            at++;
          }
        }
        pos += __shfl_sync(0xffffffffu, incl, 31);
      }
    } else if constexpr (COUNT) {
      int cnt = 0;
      for (int w = threadIdx.x; w < words; w += kSpThreads) cnt += __popc(bitmap[w]);
      int total;
      block_exclusive_scan(cnt, s_warp, &total);
      if (threadIdx.x == 0) a.row_nnz[r] = total;
    } else if constexpr (DENSE) {
      // the touched columns straight into the dense row (the rest holds the identity)
      float* drow = a.dense_u8 ? nullptr : a.dense + (long long)r * a.ldd;
      uint8_t* brow = a.dense_u8 ? a.dense_u8 + (long long)r * a.ldd : nullptr;
      for (int w = threadIdx.x; w < words; w += kSpThreads) {
        uint32_t bits = bitmap[w];
        while (bits) {
          const int j = (w << 5) + __ffs(bits) - 1;
          bits &= bits - 1;
          const float v = result(j);
          if (brow) brow[j] = 1;
          else drow[j] = v;
        }
      }
    } else {
      // columns in increasing order: word w's set bits land after all set bits of words < w
      long long out = a.dp[r];
      const long long out_end = min((long long)a.dp[r + 1], a.d_cap);
      for (int w0 = 0; w0 < words; w0 += kSpThreads) {
        const int w = w0 + threadIdx.x;
        uint32_t bits = w < words ? bitmap[w] : 0u;
        int total;
        long long pos = out + block_exclusive_scan(__popc(bits), s_warp, &total);
        while (bits) {
          const int b = __ffs(bits) - 1;
          bits &= bits - 1;
          const int j = (w << 5) + b;
          const float v = result(j);
          if (pos >= 0 && pos < out_end) {
            a.dj[pos] = j;
            a.dv[pos] = v;
          }
          pos++;
        }
        out += total;
      }
    }
    __syncthreads();  // bitmap, s_row and the scratch are reused for the next row
  }
}

// CSR structure check: rowptr[0] == 0, rowptr[rows] == nnz, offsets
// nondecreasing, columns in [0, ncols) and strictly increasing within a row.
// Sets *bad on any violation.  One warp per row, its lanes over the row's
// entries, each comparing its column with the one before it.
__global__ void csr_check_kernel(int rows, int ncols, const int* __restrict__ rp, const int* __restrict__ cj, int nnz,
                                 int* __restrict__ bad) {
  int b = 0;
  const int lane = threadIdx.x & 31;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  if (gw == 0 && lane == 0 && (rp[0] != 0 || rp[rows] != nnz)) b = 1;
  for (long long r = gw; r < rows; r += nw) {
    const int s0 = rp[r], s1 = rp[r + 1];
    if (s1 < s0 || s0 < 0 || s1 > nnz) {  // uniform across the warp
      b = 1;
      continue;
    }
    for (int e = s0 + lane; e < s1; e += 32) {
      const int j = cj[e];
      const int prev = e > s0 ? cj[e - 1] : -1;
      if (j <= prev || j >= ncols) b = 1;
    }
  }
  if (__any_sync(0xffffffffu, b) && lane == 0) atomicOr(bad, 1);
}

// Exclusive prefix sum of counts[0..n) into out[0..n], one block of 1024
// threads, each over a contiguous chunk of counts: chunk sums, one block
// scan of them, then each thread writes its chunk.  *total receives the
// exact sum, *overflow is set when it exceeds INT32 range (the offsets from
// there on hold INT32_MAX).
__global__ void __launch_bounds__(1024) offsets_scan_kernel(const int* __restrict__ counts, int n,
                                                            int* __restrict__ out, int* __restrict__ overflow,
                                                            long long* __restrict__ total) {
  __shared__ long long s_part[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int chunk = (n + 1023) / 1024;
  const long long b0 = (long long)threadIdx.x * chunk;
  const long long b1 = min((long long)n, b0 + chunk);
  long long sum = 0;
  for (long long i = b0; i < b1; i++) sum += counts[i];
  long long v = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) s_part[warp] = v;
  __syncthreads();
  long long base = 0, tot = 0;
  for (int w = 0; w < 32; w++) {
    const long long t = s_part[w];
    if (w < warp) base += t;
    tot += t;
  }
  long long run = base + v - sum;
  for (long long i = b0; i < b1; i++) {
    out[i] = run > 0x7fffffffLL ? 0x7fffffff : (int)run;
    run += counts[i];
  }
  if (threadIdx.x == 0) {
    out[n] = tot > 0x7fffffffLL ? 0x7fffffff : (int)tot;
    if (tot > 0x7fffffffLL) *overflow = 1;
    *total = tot;
  }
}

// out = 1 when the two value arrays (same structure) differ bitwise.
__global__ void values_differ_kernel(const float* __restrict__ x, const float* __restrict__ y, long long n,
                                     int* __restrict__ out) {
  int d = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    if (__float_as_uint(x[t]) != __float_as_uint(y[t])) d = 1;
  if (__any_sync(0xffffffffu, d) && (threadIdx.x & 31) == 0) atomicOr(out, 1);
}

// Dense [rows][ld] <- CSR entries (the rest was filled with the identity
// before); one warp per row.
__global__ void csr_scatter_kernel(int rows, const int* __restrict__ rp, const int* __restrict__ cj,
                                   const float* __restrict__ cv, float* __restrict__ X, long long ld) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5)
    for (int e = rp[r] + lane; e < rp[r + 1]; e += 32) X[(long long)r * ld + cj[e]] = cv[e];
}

// colcnt[j] += 1 for every stored column j (colcnt zeroed before).
__global__ void csr_col_count_kernel(const int* __restrict__ cj, long long nnz, int ncols, int* __restrict__ colcnt) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
    const int j = cj[e];
    if ((unsigned)j < (unsigned)ncols) atomicAdd(&colcnt[j], 1);
  }
}

// *out += sum_k rowcnt(k) * colcnt(k): the products a Gustavson A (x) A forms
// (each stored A[i][k] meets each stored A[k][j]).  *out zeroed before.
__global__ void csr_products_kernel(int n, const int* __restrict__ rp, const int* __restrict__ colcnt,
                                    unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    s += (unsigned long long)(rp[k + 1] - rp[k]) * (unsigned long long)colcnt[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// Entries of each dense row that differ bitwise from the identity; one warp per row.
__global__ void dense_row_count_kernel(int rows, int cols, const float* __restrict__ X, long long ld, float ident,
                                       int* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const uint32_t id = __float_as_uint(ident);
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
    int c = 0;
    for (int j = lane; j < cols; j += 32) c += __float_as_uint(X[(long long)r * ld + j]) != id;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[r] = c;
  }
}

// Per row of a byte matrix: the nonzero entries (counts[r]); *non01 = 1 when
// a byte other than 0 / 1 occurs.  One warp per row, 16 bytes per lane (one
// 16-byte load where the pitch and base allow, else byte loads).
__global__ void dense_row_count_u8_kernel(int rows, int cols, const uint8_t* __restrict__ X, long long ld,
                                          int* __restrict__ counts, int* __restrict__ non01) {
  const int lane = threadIdx.x & 31;
  const bool vec = (ld % 16 == 0) && (reinterpret_cast<uintptr_t>(X) % 16 == 0);
  uint32_t bad = 0;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
    const uint8_t* xr = X + (long long)r * ld;
    int c = 0;
    for (int j = 16 * lane; j < cols; j += 512) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      if (vec && j + 16 <= cols) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(xr + j));
        w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
      } else {
        for (int e = 0; e < 16 && j + e < cols; e++) w[e >> 2] |= (uint32_t)xr[j + e] << (8 * (e & 3));
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        c += __popc(bytes_nonzero_01(w[q]));
        bad |= w[q] & 0xfefefefeu;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[r] = c;
  }
  if (__any_sync(0xffffffffu, bad != 0) && lane == 0) atomicOr(non01, 1);
}

// CSR (values 1.0f) <- the nonzero bytes of a 0/1 byte matrix at the offsets
// rp, increasing column; one warp per row, 16 bytes per lane (as above).
__global__ void dense_to_csr_u8_kernel(int rows, int cols, const uint8_t* __restrict__ X, long long ld,
                                       const int* __restrict__ rp, int* __restrict__ cj, float* __restrict__ cv) {
  const int lane = threadIdx.x & 31;
  const bool vec = (ld % 16 == 0) && (reinterpret_cast<uintptr_t>(X) % 16 == 0);
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
    const uint8_t* xr = X + (long long)r * ld;
    int pos = rp[r];
    for (int j0 = 0; j0 < cols; j0 += 512) {
      const int j = j0 + 16 * lane;
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      if (j < cols) {
        if (vec && j + 16 <= cols) {
          const uint4 v = __ldg(reinterpret_cast<const uint4*>(xr + j));
          w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
        } else {
          for (int e = 0; e < 16 && j + e < cols; e++) w[e >> 2] |= (uint32_t)xr[j + e] << (8 * (e & 3));
        }
      }
      int c = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        w[q] = bytes_nonzero_01(w[q]);
        c += __popc(w[q]);
      }
      if (__ballot_sync(0xffffffffu, c != 0) == 0u) continue;  // uniform: no entry in these 512 columns
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      int at = pos + incl - c;
#pragma unroll
      for (int e = 0; e < 16; e++)
        if ((w[e >> 2] >> (8 * (e & 3))) & 1u) {
          cj[at] = j + e;
          cv[at] = 1.0f;
          at++;
        }
      pos += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
}

// Byte matrix entries <- 1 at the CSR's stored columns (the rest was zeroed before).
__global__ void csr_scatter_u8_kernel(int rows, const int* __restrict__ rp, const int* __restrict__ cj,
                                      uint8_t* __restrict__ X, long long ld) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5)
    for (int e = rp[r] + lane; e < rp[r + 1]; e += 32) X[(long long)r * ld + cj[e]] = 1;
}

// CSR <- dense rows (entries that are not the identity, increasing column),
// at the offsets rp; one warp per row, ballot compaction.
__global__ void dense_to_csr_kernel(int rows, int cols, const float* __restrict__ X, long long ld, float ident,
                                    const int* __restrict__ rp, int* __restrict__ cj, float* __restrict__ cv) {
  const int lane = threadIdx.x & 31;
  const uint32_t id = __float_as_uint(ident);
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
    int pos = rp[r];
    for (int j0 = 0; j0 < cols; j0 += 32) {
      const int j = j0 + lane;
      const float v = j < cols ? X[(long long)r * ld + j] : ident;
      const bool keep = j < cols && __float_as_uint(v) != id;
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int at = pos + __popc(m & ((1u << lane) - 1));
        cj[at] = j;
        cv[at] = v;
      }
      pos += __popc(m);
    }
  }
}

}  // namespace simd2
