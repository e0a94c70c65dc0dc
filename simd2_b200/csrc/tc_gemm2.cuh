// tc_gemm2.cuh -- the tensor-core srgemm on SM pairs (tcgen05 cta_group::2).
//
// A cluster of two CTAs (one per SM of a pair) computes 256 x 256 tiles of D
// with M = 256 MMAs: CTA r of the pair holds rows 128r..128r+127 of the A
// tile and rows 128r..128r+127 of the B^T tile (columns of D) in its shared
// memory, and TMEM accumulator rows for its own 128 rows of D across all 256
// columns.  Per k step each SM therefore stages 128 + 128 operand rows
// instead of 128 + 256 (tc_gemm.cuh), a third less shared-memory and L2
// traffic per MMA.
//
// Roles (both CTAs run 6 warps):
//   warp 0 lane 0 -- TMA producer of this CTA's halves (no multicast).  The
//                    transaction bytes of both CTAs complete on the even
//                    CTA's stage barrier (cp.async.bulk.tensor .cta_group::2),
//                    whose producer announces both halves' bytes,
//   warp 1 lane 0 -- (even CTA only) MMA issuer: tcgen05.mma.cta_group::2,
//                    commits multicast to both CTAs' stage-free and
//                    accumulator-full barriers,
//   warps 2..5    -- epilogue of this CTA's 128 rows (the tc_gemm.cuh tile
//                    epilogue), releasing the accumulator on the even CTA's
//                    barrier (remote arrive from the odd CTA).
// Every wait is bounded; every path ends at one cluster barrier, so neither
// CTA leaves while its peer may still signal it.
//
// Tail split: with T tiles on P pairs the last round holds r = T mod P tiles.
// When 2r <= P those r tiles run as 2r half tiles of 256 x 128 (MMA N = 128;
// each CTA loads a 64-row B box through the tmBh maps), so the last round
// takes about half a tile's time: 4096^2 on 74 pairs is 3.5 rounds of work
// instead of 4.
#pragma once
#include "common.cuh"
#include "tc_gemm.cuh"

namespace simd2 {

constexpr int kTc2BM = 256;      // rows of D per pair tile
constexpr int kTc2Stages = 6;

template <int KIND>
__host__ __device__ constexpr int tc2_half_tile() { return 128 * TcCfg<KIND>::kRowBytes; }
template <int KIND>
__host__ __device__ constexpr int tc2_stage_bytes() {
  return (TcCfg<KIND>::kNumA + TcCfg<KIND>::kNumB) * tc2_half_tile<KIND>();
}
template <int KIND>
constexpr size_t tc2_smem_bytes() {
  return (size_t)kTc2Stages * tc2_stage_bytes<KIND>() + (size_t)kTcEpiWarps * 32 * 33 * 4 + 1024 + 256;
}
// instruction descriptor: TcCfg's with M = 256 and N = n
template <int KIND>
__host__ __device__ constexpr uint32_t tc2_idesc(int n = kTcBN) {
  return (TcCfg<KIND>::kIdesc & ~(0x1Fu << 24) & ~(0x3Fu << 17)) | ((uint32_t)(kTc2BM >> 4) << 24) |
         ((uint32_t)(n >> 3) << 17);
}

__device__ __forceinline__ uint32_t cluster_rank2() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// shared::cluster address of the same shared-memory offset in CTA `rank`
__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// 2D tiled load into this CTA's shared memory, completing on the mbarrier at
// a shared::cluster address (the even CTA's), as the pair's loads do.
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t mbar_cluster, int x,
                                                 int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(mbar_cluster), "r"(x), "r"(y)
      : "memory");
}
template <int KIND>
__device__ __forceinline__ void tc2_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate,
                                        uint32_t idesc) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0),
        "r"(0));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0),
        "r"(0));
  }
}
// arrive on `bar` (same offset) in both CTAs of the pair once the issued MMAs complete
__device__ __forceinline__ void tc2_commit_both(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((unsigned short)0x3)
      : "memory");
}

template <int KIND>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_gemm2_kernel(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmA1,
                    const __grid_constant__ CUtensorMap tmB0, const __grid_constant__ CUtensorMap tmB1,
                    const __grid_constant__ CUtensorMap tmBh0, const __grid_constant__ CUtensorMap tmBh1, int M, int N,
                    int K, TcEpilogue ep, int tiles_m, int tiles_n) {
  using Cfg = TcCfg<KIND>;
  constexpr int S = kTc2Stages;
  constexpr int kStage = tc2_stage_bytes<KIND>();
  constexpr int kHalf = tc2_half_tile<KIND>();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint32_t* epi_smem = reinterpret_cast<uint32_t*>(smem + S * kStage);
  uint64_t* full = reinterpret_cast<uint64_t*>(epi_smem + kTcEpiWarps * 32 * 33);
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* fin = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);

  const uint32_t rank = cluster_rank2();
  const int pair = blockIdx.x >> 1, pairs = gridDim.x >> 1;
  const int tiles = tiles_m * tiles_n;  // 256 x 256 tiles
  const int ktiles = (K + Cfg::kBK - 1) / Cfg::kBK;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  auto tile_origin = [&](int t, int& m0, int& n0) {
    const int group = 8;
    const int per_group = group * tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gsize = min(tiles_m - first_m, group);
    const int local = t - g * per_group;
    m0 = (first_m + local % gsize) * kTc2BM;
    n0 = (local / gsize) * kTcBN;
  };
  // work items: the first `whole` tiles, then the tail's tiles as half tiles
  const int rem = tiles % pairs;
  const bool split_tail = rem > 0 && 2 * rem <= pairs;
  const int whole = split_tail ? tiles - rem : tiles;
  const int items = split_tail ? whole + 2 * rem : tiles;
  auto item_origin = [&](int w, int& m0, int& n0, int& ncols) {
    if (w < whole) {
      tile_origin(w, m0, n0);
      ncols = kTcBN;
    } else {
      const int h = w - whole;
      tile_origin(whole + (h >> 1), m0, n0);
      n0 += (h & 1) * (kTcBN / 2);
      ncols = kTcBN / 2;
    }
  };

  // Delta steps (or_and closure): every role skips the same items, an item
  // whose tile row and tile column both stayed unchanged in the previous step.
  auto skip_item = [&](int w) -> bool {
    if (!ep.need_row) return false;
    int m0, n0, ncols;
    item_origin(w, m0, n0, ncols);
    return !ep.need_row[m0 / kTc2BM] && !ep.need_col[n0 / kTcBN];
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);   // used on the even CTA: its producer's expect_tx
      mbar_init(&empty[s], 1);  // one multicast commit per use
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 2 * kTcEpiWarps);  // used on the even CTA: both CTAs' epilogue warps
    }
    mbar_init(fin, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  cluster_barrier();  // barriers initialised in both CTAs before any cross-CTA signal
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer of this CTA's halves ----------------
      prefetch_tensormap(&tmA0);
      prefetch_tensormap(&tmB0);
      prefetch_tensormap(&tmBh0);
      int j = 0;
      bool ok = true;
      for (int t = pair; t < items && ok; t += pairs) {
        if (skip_item(t)) continue;
        int m0, n0, ncols;
        item_origin(t, m0, n0, ncols);
        // this CTA's ncols/2 rows of B^T: a 128-row box, or 64 rows for a half tile
        const bool half = ncols != kTcBN;
        const CUtensorMap* mb0 = half ? &tmBh0 : &tmB0;
        const CUtensorMap* mb1 = half ? &tmBh1 : &tmB1;
        const uint32_t bytes = 2 * (Cfg::kNumA * kHalf + Cfg::kNumB * (half ? kHalf / 2 : kHalf));
        const int ma = m0 + (int)rank * 128, nb = n0 + (int)rank * (ncols / 2);
        for (int kt = 0; kt < ktiles; kt++, j++) {
          const int s = j % S;
          if (!mbar_wait(&empty[s], ((j / S) & 1) ^ 1)) {
            report_timeout(121);
            ok = false;
            break;
          }
          if (rank == 0) mbar_arrive_expect_tx(&full[s], bytes);
          const uint32_t bar0 = map_to_rank(&full[s], 0);
          uint8_t* st = smem + s * kStage;
          const int kx = kt * Cfg::kBK;
          tma_load_2d_pair(st, &tmA0, bar0, kx, ma);
          if constexpr (Cfg::kNumA == 2) tma_load_2d_pair(st + kHalf, &tmA1, bar0, kx, ma);
          uint8_t* sb = st + Cfg::kNumA * kHalf;
          tma_load_2d_pair(sb, mb0, bar0, kx, nb);
          if constexpr (Cfg::kNumB == 2) tma_load_2d_pair(sb + kHalf, mb1, bar0, kx, nb);
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------- MMA issuer of the pair ----------------
      int j = 0;
      bool ok = true;
      int lt = 0;
      // lt counts the items this pair processes (skipped ones excepted): the
      // accumulator parity and barrier phases follow it
      for (int t = pair; t < items && ok; t += pairs) {
        if (skip_item(t)) continue;
        const int acc = lt & 1;
        const uint32_t idesc = t < whole ? tc2_idesc<KIND>() : tc2_idesc<KIND>(kTcBN / 2);
        if (!mbar_wait(&acc_empty[acc], ((lt >> 1) & 1) ^ 1)) {
          report_timeout(124);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + acc * kTcBN;
        for (int kt = 0; kt < ktiles; kt++, j++) {
          const int s = j % S;
          if (!mbar_wait(&full[s], (j / S) & 1)) {
            report_timeout(122);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + s * kStage);
          const uint32_t a0 = st, a1 = st + kHalf;
          const uint32_t b0 = st + Cfg::kNumA * kHalf, b1 = b0 + kHalf;
          constexpr int RB = Cfg::kRowBytes;
#pragma unroll
          for (int ks = 0; ks < Cfg::kBK / Cfg::kKStep; ks++) {
            const uint32_t koff = ks * Cfg::kKStep * (KIND == 0 ? 2 : 1);
            const uint32_t acc0 = (kt > 0 || ks > 0) ? 1u : 0u;
            if constexpr (KIND == 0) {
              tc2_mma<0>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b0 + koff, RB), acc0, idesc);
              tc2_mma<0>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b1 + koff, RB), 1u, idesc);
              tc2_mma<0>(d, umma_desc_swizzled(a1 + koff, RB), umma_desc_swizzled(b0 + koff, RB), 1u, idesc);
            } else {
              tc2_mma<1>(d, umma_desc_swizzled(a0 + koff, RB), umma_desc_swizzled(b0 + koff, RB), acc0, idesc);
            }
          }
          tc2_commit_both(&empty[s]);  // stage s free in both CTAs once these MMAs have read it
        }
        if (ok) tc2_commit_both(&acc_full[acc]);
        lt++;
      }
      tc2_commit_both(fin);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue of this CTA's 128 rows ----------------
    const int quad = warp & 3;
    uint32_t* epi_tile = epi_smem + (warp - 2) * (32 * 33);
    bool ok = true;
    int lt = 0;
    for (int t = pair; t < items; t += pairs) {
      if (skip_item(t)) continue;
      const int acc = lt & 1;
      if (ok && !mbar_wait(&acc_full[acc], (lt >> 1) & 1)) {
        report_timeout(123);
        ok = false;
      }
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      int m0, n0, ncols;
      item_origin(t, m0, n0, ncols);
      const uint32_t trow = tmem + acc * kTcBN + ((uint32_t)(quad * 32) << 16);
      const int row0 = m0 + (int)rank * 128 + quad * 32;
      int changed = 0;
      tc_tile_epilogue<KIND>(ep, M, N, n0, row0, trow, epi_tile, lane, changed, ncols);
      if (ep.changed && KIND == 1) {
        const bool any = __any_sync(0xffffffffu, changed);
        if (any && lane == 0) {
          atomicOr(ep.changed, 1);
          if (ep.chg_row) {  // every writer stores 1
            ep.chg_row[m0 / kTc2BM] = 1;
            ep.chg_col[n0 / kTcBN] = 1;
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(map_to_rank(&acc_empty[acc], 0));
      lt++;
    }
  }

  // every MMA of the pair has completed before TMEM is released
  if (warp == 0) {
    if (!mbar_wait(fin, 0)) report_timeout(125);
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  cluster_barrier();  // no CTA leaves while its peer may still signal it
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace simd2
