// knn_fused.cuh -- k-NN with the distance block never written to memory.
//
// The materialised path (knn.cuh) writes the Q x R squared-distance matrix
// with the tensor-core minus_square kernel and reads it back for selection:
// 2 x 4 bytes of HBM traffic per (query, reference) pair.  Here the top-k
// selection runs in the epilogue of the distance MMA, so a pair costs no HBM
// traffic at all; what remains is reading the reference points (BF16 hi/lo,
// from L2 after the first CTA touches them) and writing k candidates per
// query and unit.
//
// Work unit = 128 queries x a chunk of reference tiles (256 references each).
// One CTA per unit, 10 warps:
//   warp 0 lane 0  -- TMA producer: the unit's query panels (BF16 hi and lo,
//                     64-element K panels, 128-byte swizzle) once, then per
//                     reference tile and K panel its hi and lo parts through
//                     a 5-deep ring of 32 KiB stages,
//   warp 1 lane 0  -- MMA issuer: per reference tile q.r ~ qh.rh + qh.rl + ql.rh
//                     (tcgen05.mma kind::f16, M=128, N=256, FP32 accumulate)
//                     into one of two TMEM accumulators (2 x 256 columns), so
//                     the MMAs of tile t+1 run while tile t is selected,
//   warps 2..9     -- selection: warp w reads TMEM lanes 32(w%4).. (its 32
//                     queries, lane = query) and half (w-2)/4 of the 256
//                     columns; each thread keeps the k smallest
//                     (distance, index) pairs of its query and column half
//                     in registers.
// Distances are formed exactly as the materialised minus_square epilogue
// forms them (|q|^2 + |r|^2 - 2 q.r with the FP64-accumulated norms rounded
// to FP32, and the exact FP32 sum_k (q_k - r_k)^2 inside the cancellation
// band), so both paths select from bit-identical values.  A candidate is
// examined only when it can matter: v < max(thr, band * (|q|^2 + max |r|^2
// over the tile)), thr = min(this list's k-th, the k-th of any finished
// earlier chunk of the same queries); everything else costs an FADD, an FFMA
// and a compare.
//
// Each unit writes, per query, two sorted lists of k (one per column half);
// knn_merge_kernel merges the 2 x chunks lists of a query by (distance,
// index) and writes the k results with their square roots.  Ties keep the
// lower reference index first, the order of apps/pld/emulation/knncuda.cu:
// 171-238 (insertion sort over increasing reference index).
#pragma once
#include "common.cuh"
#include "knn.cuh"
#include "prep.cuh"
#include "tc_gemm.cuh"

namespace simd2 {

constexpr int kKfBM = 128;                     // queries per unit (TMEM lanes)
constexpr int kKfBN = 256;                     // references per tile (MMA N)
constexpr int kKfMaxPanels = 2;                // D <= 128: two 64-element K panels
constexpr int kKfStages = 5;                   // B ring depth (2.5 K panels of hi + lo)
constexpr int kKfATile = kKfBM * 128;          // 16 KiB: one K panel of 128 query rows
constexpr int kKfBTile = kKfBN * 128;          // 32 KiB: one K panel of 256 reference rows
constexpr int kKfEpiWarps = 8;
constexpr int kKfThreads = (2 + kKfEpiWarps) * 32;
constexpr int kKfTmemCols = 512;               // two 128 x 256 FP32 accumulators
constexpr size_t kKfSmemBytes =
    (size_t)kKfMaxPanels * 2 * kKfATile + (size_t)kKfStages * kKfBTile + 1024 /* align */ + 256 /* barriers */;

struct KnnFusedArgs {
  int Q, R, D;
  int panels;             // ceil(round_up(D, 8) / 64), 1 or 2
  int chunks;             // reference chunks (units per 128 queries), the pilot included
  int tiles_per_chunk;    // reference tiles of 256 per chunk (after the pilot)
  int pilot_tiles;        // > 0: chunk 0 is a short pilot of this many tiles (see knn_unit_tiles)
  int num_tiles;          // ceil(R / 256)
  const float* norm_q;    // [Q]
  const float* norm_r;    // [num_tiles * 256], +inf past R
  const float* tile_nrmax;// [num_tiles]: max |r|^2 over the tile's valid references
  const float* q32;       // FP32 queries (exact recompute), row pitch ldq
  long long ldq;
  const float* r32;       // FP32 references, row pitch ldr
  long long ldr;
  float band;
  float* part_d;          // [Q][2 * chunks][K]
  int32_t* part_i;
  unsigned* ready;        // [query blocks][chunks]: 1 once the unit's lists are written (zeroed per call)
  int kout;               // neighbours asked for, at most 2K (K < kout: half-length lists, see knn_fused)
  const int* gate;        // nullable: a query block whose gate[block] is 0 is skipped (the second pass)
};

// 32-way register select by a runtime index: a 5-level tree of selects, so
// the array stays in registers.
__device__ __forceinline__ uint32_t pick32(const uint32_t (&r)[32], int j) {
  uint32_t a[16], b[8], c[4], d[2];
#pragma unroll
  for (int i = 0; i < 16; i++) a[i] = (j & 1) ? r[2 * i + 1] : r[2 * i];
#pragma unroll
  for (int i = 0; i < 8; i++) b[i] = (j & 2) ? a[2 * i + 1] : a[2 * i];
#pragma unroll
  for (int i = 0; i < 4; i++) c[i] = (j & 4) ? b[2 * i + 1] : b[2 * i];
#pragma unroll
  for (int i = 0; i < 2; i++) d[i] = (j & 8) ? c[2 * i + 1] : c[2 * i];
  return (j & 16) ? d[1] : d[0];
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Reference tiles [t0, t0 + ntiles) of a chunk.  With a pilot, chunk 0 is
// the first pilot_tiles tiles: its units are the first of the grid and run
// only a few tiles, so every later unit of the query block soon has a pruning
// bound (the units of the first wave otherwise start with none, and the first
// tiles of a list without a bound take most of the insertions).
__device__ __forceinline__ void knn_unit_tiles(const KnnFusedArgs& a, int chunk, int* t0, int* ntiles) {
  if (a.pilot_tiles > 0) {
    *t0 = chunk == 0 ? 0 : a.pilot_tiles + (chunk - 1) * a.tiles_per_chunk;
    *ntiles = min(a.num_tiles, chunk == 0 ? a.pilot_tiles : *t0 + a.tiles_per_chunk) - *t0;
  } else {
    *t0 = chunk * a.tiles_per_chunk;
    *ntiles = min(a.num_tiles, *t0 + a.tiles_per_chunk) - *t0;
  }
}

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Pruning bound from the finished units of earlier chunks of this query
// block (the four before this one, and the pilot): each of their lists holds
// K pairs no larger than its last distance, all at lower reference indices
// than this chunk's, so a candidate of this chunk at or above that distance
// is outranked K times and cannot be selected.  The bound taken from a chunk
// is the K-th smallest distance of its two lists together (K pairs at lower
// indices), tighter than the smaller of the two lists' K-th.
//
// The ready flags of those (at most five) chunks are read with relaxed loads,
// all in flight together, and only a chunk seen ready for the first time
// (bit c of *seen: chunk - 1 - c, bit 4: the pilot) costs a fence -- which,
// after the flag read, orders the list loads after the writer's release --
// and the loads of its two lists.  knn_prior_flags issues the flag loads,
// knn_prior_fold folds the newly ready chunks into the bound.
__device__ __forceinline__ void knn_prior_flags(const KnnFusedArgs& a, int qblock, int chunk, unsigned (&f)[5]) {
  const unsigned* flags = a.ready + (long long)qblock * a.chunks;
  const int lo = max(0, chunk - 4);
  const bool pilot = a.pilot_tiles > 0 && lo > 0;
#pragma unroll
  for (int c = 0; c < 4; c++) f[c] = chunk - 1 - c >= lo ? ld_relaxed_gpu(flags + chunk - 1 - c) : 0u;
  f[4] = pilot ? ld_relaxed_gpu(flags) : 0u;
}

// Folds the lists of the chunks that f shows ready and *seen does not yet
// hold into the bound T.
template <int K>
__device__ __forceinline__ float knn_prior_fold(const KnnFusedArgs& a, int chunk, int row, float T, unsigned* seen,
                                                const unsigned (&f)[5]) {
  unsigned fresh = 0;
#pragma unroll
  for (int c = 0; c < 5; c++) fresh |= (f[c] != 0u ? 1u : 0u) << c;
  fresh &= ~*seen;
  if (fresh) {
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    *seen |= fresh;
#pragma unroll
    for (int c = 0; c < 5; c++) {
      if (fresh & (1u << c)) {
        // A rank-r distance of the chunk's two sorted lists together, r >= kout:
        // the K-th smallest, min over i of max(A[i-1], B[K-1-i]) (A[-1] =
        // B[-1] = -inf), when the lists are at least kout long; with half-length
        // lists (K < kout <= 2K) the 2K-th, max(A[K-1], B[K-1]).
        const int cc = c < 4 ? chunk - 1 - c : 0;
        const float4* pa = reinterpret_cast<const float4*>(a.part_d + ((long long)row * (2 * a.chunks) + 2 * cc) * K);
        float la[K], lb[K];
#pragma unroll
        for (int u = 0; u < K / 4; u++) {
          const float4 x = __ldcg(pa + u), y = __ldcg(pa + K / 4 + u);
          la[4 * u] = x.x, la[4 * u + 1] = x.y, la[4 * u + 2] = x.z, la[4 * u + 3] = x.w;
          lb[4 * u] = y.x, lb[4 * u + 1] = y.y, lb[4 * u + 2] = y.z, lb[4 * u + 3] = y.w;
        }
        float kth;
        if (a.kout <= K) {
          kth = fminf(lb[K - 1], la[K - 1]);
#pragma unroll
          for (int i = 1; i < K; i++) kth = fminf(kth, fmaxf(la[i - 1], lb[K - 1 - i]));
        } else {
          kth = fmaxf(la[K - 1], lb[K - 1]);
        }
        T = fminf(T, kth);
      }
    }
  }
  return T;
}

template <int K>
__global__ void __launch_bounds__(kKfThreads, 1)
    knn_fused_kernel(const __grid_constant__ CUtensorMap tmQh, const __grid_constant__ CUtensorMap tmQl,
                     const __grid_constant__ CUtensorMap tmRh, const __grid_constant__ CUtensorMap tmRl,
                     KnnFusedArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;                                    // [panel][hi, lo] 16 KiB each
  uint8_t* sB = smem + kKfMaxPanels * 2 * kKfATile;      // [stage] 32 KiB each
  uint64_t* a_full = reinterpret_cast<uint64_t*>(sB + kKfStages * kKfBTile);
  uint64_t* full = a_full + 1;
  uint64_t* empty = full + kKfStages;
  uint64_t* acc_full = empty + kKfStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* fin = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);

  // chunk-major unit order: the CTAs resident at one time share reference chunks in L2
  const int qblocks = (a.Q + kKfBM - 1) / kKfBM;
  const int chunk = blockIdx.x / qblocks;
  const int m0 = (blockIdx.x - chunk * qblocks) * kKfBM;
  // second pass: only the query blocks the merge flagged
  if (a.gate && a.gate[m0 / kKfBM] == 0) return;
  int t0, ntiles;
  knn_unit_tiles(a, chunk, &t0, &ntiles);
  const int P = a.panels;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    mbar_init(a_full, 1);
    for (int s = 0; s < kKfStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < 2; s++) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], kKfEpiWarps);
    }
    mbar_init(fin, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kKfTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer ----------------
      prefetch_tensormap(&tmQh);
      prefetch_tensormap(&tmRh);
      mbar_arrive_expect_tx(a_full, 2 * P * kKfATile);
      for (int p = 0; p < P; p++) {
        tma_load_2d(sA + (2 * p) * kKfATile, &tmQh, a_full, p * 64, m0);
        tma_load_2d(sA + (2 * p + 1) * kKfATile, &tmQl, a_full, p * 64, m0);
      }
      int j = 0;
      bool ok = true;
      for (int t = 0; t < ntiles && ok; t++) {
        const int n0 = (t0 + t) * kKfBN;
        for (int p = 0; p < P && ok; p++) {
          for (int h = 0; h < 2; h++, j++) {  // panel p: hi stage, then lo stage
            const int s = j % kKfStages;
            if (!mbar_wait(&empty[s], ((j / kKfStages) & 1) ^ 1)) {
              report_timeout(111);
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&full[s], kKfBTile);
            tma_load_2d(sB + s * kKfBTile, h == 0 ? &tmRh : &tmRl, &full[s], p * 64, n0);
          }
        }
      }
    }
    __syncwarp();  // lanes 1..31 wait here, off the issue slots, while lane 0 runs the loop
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer ----------------
      bool ok = mbar_wait(a_full, 0);
      if (!ok) report_timeout(112);
      tc_fence_after();
      const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
      int j = 0;
      for (int t = 0; t < ntiles && ok; t++) {
        const int acc = t & 1;
        if (!mbar_wait(&acc_empty[acc], ((t >> 1) & 1) ^ 1)) {
          report_timeout(113);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + acc * kKfBN;
        for (int p = 0; p < P; p++, j += 2) {
          // stages j (hi) and j+1 (lo) hold K panel p of the tile
          const int sh = j % kKfStages, sl = (j + 1) % kKfStages;
          if (!mbar_wait(&full[sh], (j / kKfStages) & 1) || !mbar_wait(&full[sl], ((j + 1) / kKfStages) & 1)) {
            report_timeout(114);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t bh = b_base + sh * kKfBTile, bl = b_base + sl * kKfBTile;
          const uint32_t ah = a_base + (2 * p) * kKfATile, al = ah + kKfATile;
          // per 16-element K step: qh.rh, qh.rl, ql.rh -- the order of the
          // materialised minus_square kernel, so the FP32 sums are identical
#pragma unroll
          for (int ks = 0; ks < 4; ks++) {
            const uint32_t ko = ks * 32;  // 16 BF16 along the 128-byte row
            tc_mma<0>(d, umma_desc_sw128(ah + ko), umma_desc_sw128(bh + ko), (p > 0 || ks > 0) ? 1u : 0u);
            tc_mma<0>(d, umma_desc_sw128(ah + ko), umma_desc_sw128(bl + ko), 1u);
            tc_mma<0>(d, umma_desc_sw128(al + ko), umma_desc_sw128(bh + ko), 1u);
          }
          tc_commit(&empty[sh]);
          tc_commit(&empty[sl]);
        }
        if (ok) tc_commit(&acc_full[acc]);
      }
      tc_commit(fin);  // every MMA issued above has completed when fin flips
    }
    __syncwarp();
  } else {
    // ---------------- selection (warps 2..9) ----------------
    const int quad = warp & 3;             // TMEM lane quadrant this warp may read
    const int half = (warp - 2) >> 2;      // column half of the 256-column tile
    const int row = m0 + quad * 32 + lane;
    const bool row_ok = row < a.Q;
    const float na = row_ok ? a.norm_q[row] : 0.f;
    const float* qrow = a.q32 + (long long)(row_ok ? row : 0) * a.ldq;
    const float inf = __int_as_float(0x7f800000);
    float bd[K];
    int bi[K];
#pragma unroll
    for (int u = 0; u < K; u++) {
      bd[u] = inf;
      bi[u] = 0x7fffffff;
    }
    bool ok = true;
    const int qblock = m0 / kKfBM;
    float prior = __int_as_float(0x7f800000);  // bound from earlier chunks' lists
    unsigned seen = 0;                          // earlier chunks already folded into it
    // The bound is refreshed every tile while the unit is young (a pilot unit
    // may finish meanwhile), then every 8 tiles.  The flags a refresh folds
    // were loaded at the refresh before it, so their latency hides behind a
    // tile's selection (tile 0 loads and folds at once); flags seen a tile
    // late only leave the bound looser meanwhile.
    unsigned pf[5] = {0u, 0u, 0u, 0u, 0u};
    const bool refreshing = row_ok && chunk > 0;
    if (refreshing) {
      knn_prior_flags(a, qblock, chunk, pf);
      prior = knn_prior_fold<K>(a, chunk, row, prior, &seen, pf);
    }
    for (int t = 0; t < ntiles; t++) {
      const int acc = t & 1;
      if (refreshing && (t < 8 || (t & 7) == 0)) {
        if (t > 0) prior = knn_prior_fold<K>(a, chunk, row, prior, &seen, pf);
        knn_prior_flags(a, qblock, chunk, pf);
      }
      if (ok && !mbar_wait(&acc_full[acc], (t >> 1) & 1)) {
        report_timeout(115);
        ok = false;
      }
      ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
      if (!ok) break;
      tc_fence_after();
      const int tile = t0 + t;
      const int cbase = tile * kKfBN + half * 128;
      // band * (|q|^2 + max |r|^2) bounds band * (|q|^2 + |r|^2) over the
      // tile (FP32 addition is monotonic), so v >= lim rules out both the
      // exact recompute and an insertion (which needs v < thr)
      const float blim = a.band * (na + a.tile_nrmax[tile]);
      float thr = fminf(bd[K - 1], prior);
      float lim = fmaxf(thr, blim);
      const uint32_t taddr = tmem + acc * kKfBN + half * 128 + ((uint32_t)(quad * 32) << 16);
#pragma unroll 1
      for (int c2 = 0; c2 < 2; c2++) {
        // 64 columns per TMEM round trip (tcgen05.ld .x64, one wait)
        uint32_t r64[64];
        tmem_ld64(taddr + c2 * 64, r64);
        if (c2 == 1) {
          // the accumulator is in registers: hand it back to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[acc]);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c = 2 * c2 + h;
          uint32_t(&r)[32] = *reinterpret_cast<uint32_t(*)[32]>(r64 + 32 * h);
          // Hot pass: the distance of each of the 32 columns and a bit per
          // column that may enter the list.  The insertion code exists once per
          // half, below, so the loop body stays small for the instruction cache.
          // Packed FP32 pairs: each lane of __fadd2_rn / __ffma2_rn rounds
          // like the scalar na + |r|^2 and fma(-2, q.r, .), so v keeps the
          // materialised epilogue's bits.
          const float4* nb4 = reinterpret_cast<const float4*>(a.norm_r + cbase + c * 32);
          const float2 na2 = make_float2(na, na), m2 = make_float2(-2.0f, -2.0f);
          // The mask bits are formed as 1.0 / 0.0 and summed with packed FMAs
          // into four accumulators of 16 bit positions each (exact: every sum
          // stays below 2^16), which leaves one compare per column on the ALU
          // pipe (the selection warps keep that pipe busy) and moves the rest
          // to the FMA pipe.
          float2 mlo = make_float2(0.f, 0.f), mhi = make_float2(0.f, 0.f);
#pragma unroll
          for (int q4 = 0; q4 < 8; q4++) {
            const float4 nb = __ldg(nb4 + q4);
#pragma unroll
            for (int e = 0; e < 4; e += 2) {
              const int jj = q4 * 4 + e;
              const float2 s2 = __fadd2_rn(na2, e == 0 ? make_float2(nb.x, nb.y) : make_float2(nb.z, nb.w));
              const float2 v2 =
                  __ffma2_rn(m2, make_float2(__uint_as_float(r[jj]), __uint_as_float(r[jj + 1])), s2);
              r[jj] = __float_as_uint(v2.x);
              r[jj + 1] = __float_as_uint(v2.y);
              const float2 b2 = make_float2(v2.x < lim ? 1.f : 0.f, v2.y < lim ? 1.f : 0.f);
              const int pos = jj & 15;
              const float2 w2 = make_float2((float)(1u << pos), (float)(2u << pos));
              if (jj < 16) mlo = __ffma2_rn(b2, w2, mlo);
              else mhi = __ffma2_rn(b2, w2, mhi);
            }
          }
          uint32_t mask = (uint32_t)(mlo.x + mlo.y) | ((uint32_t)(mhi.x + mhi.y) << 16);
          // Rare pass, in increasing column order.
          while (mask) {
            const int j = __ffs(mask) - 1;
            mask &= mask - 1;
            const int col = cbase + c * 32 + j;
            float v = __uint_as_float(pick32(r, j));
            // blim >= band * (|q|^2 + |r|^2) for every column of the tile, so
            // only v < blim can be in the cancellation band
            if (v < blim && v < a.band * (na + a.norm_r[col])) v = exact_minus_square(qrow, a.r32, a.ldr, col, a.D, 1);
            if (v < thr) {
              topk_insert<K>(bd, bi, v, col);
              thr = fminf(bd[K - 1], prior);
              lim = fmaxf(thr, blim);
            }
          }
        }
      }
    }
    if (row_ok) {
      const long long base = ((long long)row * (2 * a.chunks) + 2 * chunk + half) * K;
#pragma unroll
      for (int u = 0; u < K; u += 4) {
        *reinterpret_cast<float4*>(a.part_d + base + u) = make_float4(bd[u], bd[u + 1], bd[u + 2], bd[u + 3]);
        *reinterpret_cast<int4*>(a.part_i + base + u) = make_int4(bi[u], bi[u + 1], bi[u + 2], bi[u + 3]);
      }
    }
    // publish: every selection thread's lists, then the unit's ready flag
    __threadfence();
    asm volatile("bar.sync 1, %0;" ::"r"(kKfEpiWarps * 32) : "memory");
    if (warp == 2 && lane == 0 && ok) st_release_gpu(a.ready + (long long)qblock * a.chunks + chunk, 1u);
  }

  // every MMA has completed before TMEM is released
  if (warp == 0) {
    if (!mbar_wait(fin, 0)) report_timeout(116);
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kKfTmemCols) : "memory");
  }
}

// Insert (v, i) into a list sorted by (distance, index); for merging lists
// whose indices arrive in no particular order.
template <int K>
__device__ __forceinline__ void topk_insert_lex(float (&bd)[K], int (&bi)[K], float v, int i) {
#pragma unroll
  for (int t = K - 1; t > 0; t--) {
    const bool shift = lex_less(v, i, bd[t - 1], bi[t - 1]);
    const bool place = !shift && lex_less(v, i, bd[t], bi[t]);
    bd[t] = shift ? bd[t - 1] : (place ? v : bd[t]);
    bi[t] = shift ? bi[t - 1] : (place ? i : bi[t]);
  }
  if (lex_less(v, i, bd[0], bi[0])) {
    bd[0] = v;
    bi[0] = i;
  }
}

// Merges each query's `lists` sorted lists of KL candidates into the kout
// smallest by (distance, index), writes their square roots and indices (-1
// where fewer than kout references exist).  K (>= kout) is the capacity of a
// lane's list.
// G = lanes per query (a power of two, 32 / G queries per warp).  When
// lists <= G, lane l of a group loads list l whole into registers (16-byte
// loads) and the group takes kout rounds of a (distance, index) argmin over
// the lanes' heads, the winner shifting its list by one.  Otherwise each lane
// first folds lists l, l+G, ... into one sorted list by insertion.
//
// flags (KL < kout, the first pass of knn_fused): a list of KL entries that
// is full may have left out candidates at or above its last entry (its unit
// pruned with its own KL-th).  Those could belong to the result only when
// that last entry precedes the result's kout-th in (distance, index) order;
// then flags[query block] is set and the block is redone with full-length
// lists.  gate (the second pass): only the query blocks with gate[block] set
// are merged and written.
template <int KL, int K, int G>
__global__ void __launch_bounds__(256) knn_merge_kernel(const float* __restrict__ part_d,
                                                        const int32_t* __restrict__ part_i, int rows, int lists,
                                                        float* __restrict__ out_d, int32_t* __restrict__ out_i,
                                                        long long ldo, int kout, int* __restrict__ flags,
                                                        const int* __restrict__ gate) {
  static_assert(KL <= K, "input lists fit a lane's list");
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  const float inf = __int_as_float(0x7f800000);
  constexpr int kGroups = 32 / G;  // queries per warp, all in one block of 128 rows
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  // the loop bound is uniform across the warp, so every lane takes the shuffles
  for (int r0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kGroups; r0 < rows; r0 += nwarps * kGroups) {
    if (gate && gate[r0 / kKfBM] == 0) continue;  // uniform across the warp
    const int r = r0 + lane / G;
    const bool live = r < rows;
    float bd[K];
    int bi[K];
#pragma unroll
    for (int t = 0; t < K; t++) {
      bd[t] = inf;
      bi[t] = 0x7fffffff;
    }
    // the smallest last entry of a full input list this lane holds
    float fl = inf;
    int fli = 0x7fffffff;
    if (live && lists <= G) {
      if (sub < lists) {
        const float4* ld = reinterpret_cast<const float4*>(part_d + ((long long)r * lists + sub) * KL);
        const int4* li = reinterpret_cast<const int4*>(part_i + ((long long)r * lists + sub) * KL);
#pragma unroll
        for (int u = 0; u < KL / 4; u++) {
          const float4 v = ld[u];
          const int4 w = li[u];
          bd[4 * u] = v.x, bd[4 * u + 1] = v.y, bd[4 * u + 2] = v.z, bd[4 * u + 3] = v.w;
          bi[4 * u] = w.x, bi[4 * u + 1] = w.y, bi[4 * u + 2] = w.z, bi[4 * u + 3] = w.w;
        }
        if (bi[KL - 1] != 0x7fffffff) {
          fl = bd[KL - 1];
          fli = bi[KL - 1];
        }
      }
    } else if (live) {
      for (int l = sub; l < lists; l += G) {
        const float* ld = part_d + ((long long)r * lists + l) * KL;
        const int32_t* li = part_i + ((long long)r * lists + l) * KL;
        const int last = li[KL - 1];
        if (last != 0x7fffffff && lex_less(ld[KL - 1], last, fl, fli)) {
          fl = ld[KL - 1];
          fli = last;
        }
        for (int e = 0; e < KL; e++) {
          const float v = ld[e];
          const int ix = li[e];
          if (!lex_less(v, ix, bd[K - 1], bi[K - 1])) break;  // the list is sorted
          topk_insert_lex<K>(bd, bi, v, ix);
        }
      }
    }
    float v = inf;
    int ix = 0x7fffffff;
    for (int t = 0; t < kout; t++) {
      v = bd[0];
      ix = bi[0];
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, ix, o);
        if (lex_less(v2, i2, v, ix)) {
          v = v2;
          ix = i2;
        }
      }
      if (bd[0] == v && bi[0] == ix) {
#pragma unroll
        for (int u = 0; u < K - 1; u++) {
          bd[u] = bd[u + 1];
          bi[u] = bi[u + 1];
        }
        bd[K - 1] = inf;
        bi[K - 1] = 0x7fffffff;
      }
      if (sub == 0 && live) {
        out_d[(long long)r * ldo + t] = sqrtf(fmaxf(v, 0.f));
        out_i[(long long)r * ldo + t] = ix == 0x7fffffff ? -1 : ix;
      }
    }
    // (v, ix) is now the kout-th result, the same in every lane of the group
    if (flags && live && lex_less(fl, fli, v, ix)) atomicOr(&flags[r / kKfBM], 1);
  }
}

// Operand preparation of the fused k-NN in one launch.  Per row of the
// queries and of the references: the squared norm in FP64 rounded to float
// (lane l adds the squares of elements l, l+32, ... in that order, then a
// butterfly over the warp: row_norms_kernel's order, so the same bits) and
// the BF16 hi / lo split in split_rows_bf16_kernel's layout ([rows][Dp],
// zeros past D).  Blocks [0, r_tiles) take one 256-reference tile each and
// also write the tile's largest norm over its valid references, and +inf
// norms for the padding references past R; the blocks after them take 256
// queries each.  The grid also clears `clear_words` words at `clear` (the
// passes' ready and block flags).  32 warps per block, 8 rows per warp: a
// warp issues all its loads at once (lane l holds elements l, l+32, ... of
// each row) and splits from the same registers.
struct KnnPrepArgs {
  const float* q;
  long long ldq;
  int Q;
  const float* r;
  long long ldr;
  int R;
  int D, Dp;  // D <= 32 * kKnnPrepMaxJ, Dp = D rounded up to 8
  __nv_bfloat16 *q_hi, *q_lo, *r_hi, *r_lo;
  float *n_q, *n_r, *t_max;
  int r_tiles;
  unsigned* clear;
  long long clear_words;
};

constexpr int kKnnPrepMaxJ = kKfMaxPanels * 2;  // D <= 128: four elements per lane and row
constexpr int kKnnPrepRows = 8;                 // rows per warp
constexpr int kKnnPrepThreads = 1024;           // 32 warps x 8 rows = 256 rows per block
static_assert(kKnnPrepThreads / 32 * kKnnPrepRows == kKfBN, "one reference tile per block");

__global__ void __launch_bounds__(kKnnPrepThreads) knn_prep_kernel(KnnPrepArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long w = blockIdx.x * (long long)kKnnPrepThreads + threadIdx.x; w < a.clear_words;
       w += (long long)gridDim.x * kKnnPrepThreads)
    a.clear[w] = 0u;
  const bool ref = blockIdx.x < a.r_tiles;
  const float* A = ref ? a.r : a.q;
  const long long lda = ref ? a.ldr : a.ldq;
  const int M = ref ? a.R : a.Q;
  const int rows = ref ? a.r_tiles * kKfBN : M;  // norms written for rows < rows
  __nv_bfloat16* hi = ref ? a.r_hi : a.q_hi;
  __nv_bfloat16* lo = ref ? a.r_lo : a.q_lo;
  float* nrm = ref ? a.n_r : a.n_q;
  const int row0 = (ref ? blockIdx.x : blockIdx.x - a.r_tiles) * kKfBN + warp * kKnnPrepRows;
  const float inf = __int_as_float(0x7f800000);
  float mx = -inf;  // the warp's largest norm over valid rows (reference tiles)
  {
    float v[kKnnPrepRows][kKnnPrepMaxJ];
#pragma unroll
    for (int u = 0; u < kKnnPrepRows; u++) {
      const int i = row0 + u;
#pragma unroll
      for (int j = 0; j < kKnnPrepMaxJ; j++) {
        const int k = lane + 32 * j;
        v[u][j] = (i < M && k < a.D) ? __ldg(A + (long long)i * lda + k) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < kKnnPrepRows; u++) {
      const int i = row0 + u;
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < kKnnPrepMaxJ; j++) {
        if (lane + 32 * j < a.D) {
          const double x = v[u][j];
          s += x * x;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const float n = i < M ? (float)s : inf;
      if (i < M) mx = fmaxf(mx, n);
      if (lane == 0 && i < rows) nrm[i] = n;
    }
    // the BF16 split from the same registers: lane l writes elements l,
    // l+32, ... of each row (zeros for D <= k < Dp)
#pragma unroll
    for (int u = 0; u < kKnnPrepRows; u++) {
      const int i = row0 + u;
      if (i >= M) continue;
#pragma unroll
      for (int j = 0; j < kKnnPrepMaxJ; j++) {
        const int k = lane + 32 * j;
        if (k < a.Dp) {
          __nv_bfloat16 h, l;
          split_bf16(v[u][j], h, l);
          hi[(long long)i * a.Dp + k] = h;
          lo[(long long)i * a.Dp + k] = l;
        }
      }
    }
  }
  if (!ref) return;  // uniform across the block
  __shared__ float wmax[kKnnPrepThreads / 32];
  if (lane == 0) wmax[warp] = mx;
  __syncthreads();
  if (warp == 0) {
    float m = wmax[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) a.t_max[blockIdx.x] = m;
  }
}

}  // namespace simd2
