// tc_gemm.cuh -- tensor-core (tcgen05 / TMEM) srgemm paths for sm_100a.
//
// Used for the semirings that are dense contractions:
//   * or_and       : kind::i8, unsigned 0/1 bytes, S32 counts; D = (count > 0) | C.
//   * plus_mul     : kind::f16 with BF16 hi/lo operands, FP32 accumulate:
//                    a*b ~= a_hi*b_hi + a_hi*b_lo + a_lo*b_hi  (three MMAs per k step).
//   * minus_square : the same BF16 hi/lo product gives a.b; the epilogue forms
//                    |a|^2 + |b|^2 - 2 a.b with FP64-accumulated norms and
//                    recomputes sum_k (a-b)^2 exactly in FP32 inside the
//                    cancellation band (small distance relative to the norms).
//
// Persistent: one CTA per SM walks the 128 x 256 tiles of D (grouped raster)
// with 6 warps:
//   warp 0 lane 0  -- TMA producer (2D tiled loads, no multicast; 64-byte
//                     swizzled rows for BF16, 128-byte for INT8) over every
//                     k-tile of every tile, one ring of stages,
//   warp 1 lane 0  -- MMA issuer (tcgen05.mma, cta_group::1, M=128 N=256) into
//                     one of two 256-column TMEM accumulators, so the next
//                     tile's MMAs run while the previous tile is written out,
//   warps 2..5     -- epilogue: tcgen05.ld of the accumulator (warp w reads
//                     TMEM lanes 32(w%4)..+31 = tile rows), fused (+) C, stores.
// Both operands are K-major in shared memory: A is [M][K] as given, B is
// stored transposed ([N][K]) by the operand-prep kernel.
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kTcBM = 128;
constexpr int kTcBN = 256;
constexpr int kTcEpiWarps = 4;
constexpr int kTcThreads = (2 + kTcEpiWarps) * 32;  // TMA warp, MMA warp, 4 epilogue warps
template <int KIND>
struct TcCfg;
// BF16 hi/lo: BK = 32 elements (64-byte swizzled rows), two A tiles and two B
// tiles per stage, 4 stages of 48 KiB: three stages stay in flight while one
// feeds the tensor cores (two 96 KiB stages of 128-byte rows left the TMA
// latency exposed).
template <>
struct TcCfg<0> {
  static constexpr int kBK = 32;
  static constexpr int kRowBytes = 64;
  static constexpr int kNumA = 2;
  static constexpr int kNumB = 2;
  static constexpr int kStages = 4;
  static constexpr int kKStep = 16;  // K per tcgen05.mma kind::f16
  // c_format F32 (1), a/b format BF16 (1), K-major A and B, N=256, M=128
  static constexpr uint32_t kIdesc =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcBN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
};
// INT8 0/1: BK = 128 elements, one A and one B tile per stage.
template <>
struct TcCfg<1> {
  static constexpr int kBK = 128;
  static constexpr int kRowBytes = 128;
  static constexpr int kNumA = 1;
  static constexpr int kNumB = 1;
  static constexpr int kStages = 4;
  static constexpr int kKStep = 32;  // K per tcgen05.mma kind::i8
  // c_format S32 (2), a/b format unsigned 8-bit (0), K-major, N=256, M=128
  static constexpr uint32_t kIdesc = (2u << 4) | ((uint32_t)(kTcBN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
};

template <int KIND>
__host__ __device__ constexpr int tc_a_tile() { return kTcBM * TcCfg<KIND>::kRowBytes; }
template <int KIND>
__host__ __device__ constexpr int tc_b_tile() { return kTcBN * TcCfg<KIND>::kRowBytes; }

template <int KIND>
__host__ __device__ constexpr int tc_stage_bytes() {
  return TcCfg<KIND>::kNumA * tc_a_tile<KIND>() + TcCfg<KIND>::kNumB * tc_b_tile<KIND>();
}
template <int KIND>
constexpr size_t tc_smem_bytes() {
  return (size_t)TcCfg<KIND>::kStages * tc_stage_bytes<KIND>() + (size_t)kTcEpiWarps * 32 * 33 * 4 + 1024 + 256;
}

// Shared-memory matrix descriptor for a K-major operand tile written by TMA
// with a 128- or 64-byte swizzle: rows of row_bytes, 8-row core-matrix groups
// 8 * row_bytes apart (stride byte offset), leading byte offset unused (1),
// version 1, layout type 2 = SWIZZLE_128B or 4 = SWIZZLE_64B.  Advancing K
// inside a row moves the start address by the byte offset.
__device__ __forceinline__ uint64_t umma_desc_swizzled(uint32_t smem_addr, int row_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                             // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8u * row_bytes) >> 4) << 32;        // stride byte offset
  d |= (uint64_t)1u << 46;                             // descriptor version (sm_100)
  d |= (uint64_t)(row_bytes == 128 ? 2u : 4u) << 61;   // SWIZZLE_128B / SWIZZLE_64B
  return d;
}

// The descriptor for 128-byte swizzled rows (8-row groups 1024 bytes apart).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr) {
  return umma_desc_swizzled(smem_addr, 128);
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

template <int KIND>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(TcCfg<0>::kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(TcCfg<1>::kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  }
}

// Arrive on `bar` once every tcgen05 operation issued so far by this thread completes.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread t of the warp gets lane t.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 lanes x 64 consecutive 32-bit columns in one round trip.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&r)[64]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
      "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
      "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
        "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
        "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Epilogue arguments of the tensor-core paths.
struct TcEpilogue {
  int op;               // SIMD2_PLUS_MUL, SIMD2_MINUS_SQUARE or SIMD2_OR_AND
  int do_epilogue;
  const void* C;        // float (sums) or int32 / uint8 (or_and)
  long long ldc;
  void* D;
  long long ldd;
  int out_u8;           // or_and: 1 = uint8 C/D, 0 = int32 C/D
  // minus_square: row norms of A (M), column norms of B (N), and the FP32
  // operands for the exact recompute inside the cancellation band.
  const float* norm_a;
  const float* norm_b;
  const float* A32;
  long long lda32;
  const float* B32;
  long long ldb32;
  int K;
  float band;           // recompute when dist < band * (|a|^2 + |b|^2)
  int b_rows;           // 1: B32 holds B transposed ([N][K], e.g. k-NN reference points)
  int* changed;         // or_and closure: set to 1 when any D differs from C
  // Delta steps of the or_and closure (tc_gemm2_kernel only): chg_row[i] /
  // chg_col[j] receive a 1 when an element of 256-row tile row i / 256-column
  // tile column j changed; with need_row / need_col (the previous step's maps)
  // a tile whose tile row and tile column both stayed unchanged is skipped --
  // every product it would form was formed in that step and is already in C.
  uint8_t* chg_row;
  uint8_t* chg_col;
  const uint8_t* need_row;
  const uint8_t* need_col;
};

// sum_k (a[k] - B[k][col])^2 in FP32; B is [K][N] (pitch ldb) or, when
// b_rows, stored transposed as [N][K].
__device__ __forceinline__ float exact_minus_square(const float* a, const float* B, long long ldb, int col, int K,
                                                    int b_rows) {
  float s = 0.f;
  if (b_rows) {
    const float* b = B + (long long)col * ldb;
    for (int k = 0; k < K; k++) {
      const float d = __fsub_rn(a[k], b[k]);
      s = __fmaf_rn(d, d, s);
    }
  } else {
    for (int k = 0; k < K; k++) {
      const float d = __fsub_rn(a[k], B[(long long)k * ldb + col]);
      s = __fmaf_rn(d, d, s);
    }
  }
  return s;
}

// Epilogue of one 128 x ncols tile (ncols = 256, or 128 for a split tail
// tile) for the 32 rows of one warp: lane l holds row row0 + l of the
// accumulator in TMEM at trow (lane quadrant and column base included).  Sets
// changed when an or_and output differs from C.
template <int KIND>
__device__ __forceinline__ void tc_tile_epilogue(const TcEpilogue& ep, int M, int N, int n0, int row0, uint32_t trow,
                                                 uint32_t* epi_tile, int lane, int& changed, int ncols = kTcBN) {
  if constexpr (KIND == 1) {
    // or_and: 32 flags of one row are 32 contiguous bytes (u8) or 128 bytes
    // (i32), so each lane writes its own row with 16-byte vector stores.
    const int row = row0 + lane;
    const bool u8 = ep.out_u8 != 0;
    const int esz = u8 ? 1 : 4;
    const bool vec_ok = ((ep.ldd * esz) % 16 == 0) && ((reinterpret_cast<uintptr_t>(ep.D) & 15) == 0) &&
                        (!ep.do_epilogue ||
                         (((ep.ldc * esz) % 16 == 0) && ((reinterpret_cast<uintptr_t>(ep.C) & 15) == 0)));
#pragma unroll 1
    for (int c0 = 0; c0 < ncols; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(trow + c0, r);  // all lanes take part (sync.aligned)
      if (row >= M) continue;
      const int colb = n0 + c0;
      if (u8) {
        const uint8_t* crow = static_cast<const uint8_t*>(ep.C) + (long long)row * ep.ldc;
        uint8_t* drow = static_cast<uint8_t*>(ep.D) + (long long)row * ep.ldd;
        if (vec_ok && colb + 32 <= N) {
          uint32_t w[8];
#pragma unroll
          for (int q = 0; q < 8; q++)
            w[q] = (r[4 * q] != 0u) | ((r[4 * q + 1] != 0u) << 8) | ((r[4 * q + 2] != 0u) << 16) |
                   ((uint32_t)(r[4 * q + 3] != 0u) << 24);
          if (ep.do_epilogue) {
            const uint4 c0v = *reinterpret_cast<const uint4*>(crow + colb);
            const uint4 c1v = *reinterpret_cast<const uint4*>(crow + colb + 16);
            const uint32_t cw[8] = {c0v.x, c0v.y, c0v.z, c0v.w, c1v.x, c1v.y, c1v.z, c1v.w};
#pragma unroll
            for (int q = 0; q < 8; q++) {
              const uint32_t cb = bytes_nonzero_01(cw[q]);  // C's bytes as 0/1 before the OR
              const uint32_t v = w[q] | cb;
              if (ep.changed && v != cb) changed = 1;
              w[q] = v;
            }
          }
          *reinterpret_cast<uint4*>(drow + colb) = make_uint4(w[0], w[1], w[2], w[3]);
          *reinterpret_cast<uint4*>(drow + colb + 16) = make_uint4(w[4], w[5], w[6], w[7]);
        } else {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const int col = colb + j;
            if (col < N) {
              uint8_t v = r[j] != 0u;
              if (ep.do_epilogue) {
                const uint8_t cv = crow[col] != 0;
                v |= cv;
                if (ep.changed && v != cv) changed = 1;
              }
              drow[col] = v;
            }
          }
        }
      } else {
        const int32_t* crow = static_cast<const int32_t*>(ep.C) + (long long)row * ep.ldc;
        int32_t* drow = static_cast<int32_t*>(ep.D) + (long long)row * ep.ldd;
        if (vec_ok && colb + 32 <= N) {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            int4 v = make_int4(r[4 * q] != 0u, r[4 * q + 1] != 0u, r[4 * q + 2] != 0u, r[4 * q + 3] != 0u);
            if (ep.do_epilogue) {
              const int4 c = *reinterpret_cast<const int4*>(crow + colb + 4 * q);
              v.x |= c.x != 0;
              v.y |= c.y != 0;
              v.z |= c.z != 0;
              v.w |= c.w != 0;
            }
            *reinterpret_cast<int4*>(drow + colb + 4 * q) = v;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const int col = colb + j;
            if (col < N) {
              int32_t v = r[j] != 0u;
              if (ep.do_epilogue) v |= (crow[col] != 0);
              drow[col] = v;
            }
          }
        }
      }
    }
  } else {
    // Sums: a 32 x 32 chunk is transposed through shared memory (the stage
    // ring is idle now) and written row by row: lane l handles column l, so
    // every store instruction covers 32 consecutive floats of one row.  The
    // chunk's C values (one column per lane, 32 independent loads) and the
    // warp's 32 row norms are fetched before the TMEM read, so their latency
    // overlaps it instead of being paid row by row.
    uint32_t* tile = epi_tile;
    const bool msq = ep.op == SIMD2_MINUS_SQUARE;
    const float na_lane = (msq && row0 + lane < M) ? ep.norm_a[row0 + lane] : 0.f;
    const int rows_here = min(32, M - row0);
#pragma unroll 1
    for (int c0 = 0; c0 < ncols; c0 += 32) {
      const int col = n0 + c0 + lane;
      const bool col_ok = col < N;
      float cv[32];
      if (ep.do_epilogue) {
        const float* Cc = static_cast<const float*>(ep.C) + col;
#pragma unroll
        for (int rr = 0; rr < 32; rr++)
          cv[rr] = (col_ok && rr < rows_here) ? Cc[(long long)(row0 + rr) * ep.ldc] : 0.f;
      }
      const float nb = (msq && col_ok) ? ep.norm_b[col] : 0.f;
      uint32_t r[32];
      tmem_ld32(trow + c0, r);  // all lanes take part (sync.aligned)
#pragma unroll
      for (int j = 0; j < 32; j++) tile[lane * 33 + j] = r[j];
      __syncwarp();
      if (msq) {
        // distances in place; rows inside the cancellation band are
        // recomputed exactly in a separate, rarely taken loop (one copy of
        // the recompute code)
        uint32_t band = 0;
#pragma unroll
        for (int rr = 0; rr < 32; rr++) {
          const float nsum = __shfl_sync(0xffffffffu, na_lane, rr) + nb;
          const float v = __fmaf_rn(-2.0f, __uint_as_float(tile[rr * 33 + lane]), nsum);
          tile[rr * 33 + lane] = __float_as_uint(v);
          band |= (v < ep.band * nsum && rr < rows_here && col_ok ? 1u : 0u) << rr;
        }
        while (band) {
          const int rr = __ffs(band) - 1;
          band &= band - 1;
          tile[rr * 33 + lane] = __float_as_uint(exact_minus_square(
              ep.A32 + (long long)(row0 + rr) * ep.lda32, ep.B32, ep.ldb32, col, ep.K, ep.b_rows));
        }
      }
      if (col_ok) {
        float* Dc = static_cast<float*>(ep.D) + col;
#pragma unroll
        for (int rr = 0; rr < 32; rr++) {
          if (rr < rows_here) {
            float v = __uint_as_float(tile[rr * 33 + lane]);
            if (ep.do_epilogue) v = __fadd_rn(v, cv[rr]);
            Dc[(long long)(row0 + rr) * ep.ldd] = v;
          }
        }
      }
      __syncwarp();
    }
  }
}
template <int KIND>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmA1,
                   const __grid_constant__ CUtensorMap tmB0, const __grid_constant__ CUtensorMap tmB1, int M, int N,
                   int K, TcEpilogue ep, int tiles_m, int tiles_n) {
  using Cfg = TcCfg<KIND>;
  constexpr int S = Cfg::kStages;
  constexpr int kStage = tc_stage_bytes<KIND>();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint32_t* epi_smem = reinterpret_cast<uint32_t*>(smem + S * kStage);  // 4 x 32 x 33 words
  uint64_t* full = reinterpret_cast<uint64_t*>(epi_smem + kTcEpiWarps * 32 * 33);
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* fin = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);

  const int tiles = tiles_m * tiles_n;
  const int ktiles = (K + Cfg::kBK - 1) / Cfg::kBK;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  // Grouped raster over (tile_m, tile_n): 8 tile rows per group.
  auto tile_origin = [&](int t, int& m0, int& n0) {
    const int group = 8;
    const int per_group = group * tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gsize = min(tiles_m - first_m, group);
    const int local = t - g * per_group;
    m0 = (first_m + local % gsize) * kTcBM;
    n0 = (local / gsize) * kTcBN;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], kTcEpiWarps);
    }
    mbar_init(fin, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    // 512 TMEM columns: two 128 x 256 FP32/S32 accumulators.
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer: every k-tile of every tile of this CTA ----------------
      prefetch_tensormap(&tmA0);
      prefetch_tensormap(&tmB0);
      int j = 0;  // running stage counter
      bool ok = true;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        int m0, n0;
        tile_origin(t, m0, n0);
        for (int kt = 0; kt < ktiles; kt++, j++) {
          const int s = j % S;
          if (!mbar_wait(&empty[s], ((j / S) & 1) ^ 1)) {
            report_timeout(101);
            ok = false;
            break;
          }
          uint8_t* st = smem + s * kStage;
          mbar_arrive_expect_tx(&full[s], kStage);
          const int kx = kt * Cfg::kBK;
          tma_load_2d(st, &tmA0, &full[s], kx, m0);
          if constexpr (Cfg::kNumA == 2) tma_load_2d(st + tc_a_tile<KIND>(), &tmA1, &full[s], kx, m0);
          uint8_t* sb = st + Cfg::kNumA * tc_a_tile<KIND>();
          tma_load_2d(sb, &tmB0, &full[s], kx, n0);
          if constexpr (Cfg::kNumB == 2) tma_load_2d(sb + tc_b_tile<KIND>(), &tmB1, &full[s], kx, n0);
        }
      }
    }
    __syncwarp();  // lanes 1..31 wait here, off the issue slots, while lane 0 runs the loop
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer: tile lt accumulates into TMEM half lt & 1 ----------------
      int j = 0;
      bool ok = true;
      int lt = 0;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, lt++) {
        const int acc = lt & 1;
        if (!mbar_wait(&acc_empty[acc], ((lt >> 1) & 1) ^ 1)) {
          report_timeout(104);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + acc * kTcBN;
        for (int kt = 0; kt < ktiles; kt++, j++) {
          const int s = j % S;
          if (!mbar_wait(&full[s], (j / S) & 1)) {
            report_timeout(102);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + s * kStage);
          const uint32_t a0 = st, a1 = st + tc_a_tile<KIND>();
          const uint32_t b0 = st + Cfg::kNumA * tc_a_tile<KIND>(), b1 = b0 + tc_b_tile<KIND>();
          constexpr int RB = Cfg::kRowBytes;
#pragma unroll
          for (int ks = 0; ks < Cfg::kBK / Cfg::kKStep; ks++) {
            const uint32_t koff = ks * Cfg::kKStep * (KIND == 0 ? 2 : 1);  // bytes along the swizzled row
            const uint32_t acc0 = (kt > 0 || ks > 0) ? 1u : 0u;
            if constexpr (KIND == 0) {
              // hi*hi, hi*lo, lo*hi
              tc_mma<0>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b0 + koff, RB), acc0);
              tc_mma<0>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b1 + koff, RB), 1u);
              tc_mma<0>(d, umma_desc_swizzled(a1 + koff, RB), umma_desc_swizzled(b0 + koff, RB), 1u);
            } else {
              tc_mma<1>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b0 + koff, RB), acc0);
            }
          }
          tc_commit(&empty[s]);  // stage s is free once these MMAs have read it
        }
        if (ok) tc_commit(&acc_full[acc]);  // accumulator complete
      }
      tc_commit(fin);  // every MMA issued above has completed when fin flips
    }
    __syncwarp();
  } else {
    // ---------------- epilogue warps 2..5: warp w reads TMEM lanes 32 (w % 4) .. ----------------
    const int quad = warp & 3;
    uint32_t* epi_tile = epi_smem + (warp - 2) * (32 * 33);
    bool ok = true;
    int lt = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, lt++) {
      const int acc = lt & 1;
      if (ok && !mbar_wait(&acc_full[acc], (lt >> 1) & 1)) {
        report_timeout(103);
        ok = false;
      }
      ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld below is warp-collective
      if (!ok) break;
      tc_fence_after();
      int m0, n0;
      tile_origin(t, m0, n0);
      const uint32_t trow = tmem + acc * kTcBN + ((uint32_t)(quad * 32) << 16);
      const int row0 = m0 + quad * 32;
      int changed = 0;
      tc_tile_epilogue<KIND>(ep, M, N, n0, row0, trow, epi_tile, lane, changed);
      if (ep.changed && KIND == 1) {
        if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(ep.changed, 1);
      }
      // the accumulator half is read out: the MMA warp may reuse it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[acc]);
    }
  }

  // every MMA has completed before TMEM is released
  if (warp == 0) {
    if (!mbar_wait(fin, 0)) report_timeout(105);
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace simd2
