// srgemm_simt.cuh -- FP32 CUDA-core semiring GEMM for sm_100a.
//
// Computes one BM x BN tile of D = id (+) A(x)B [(+) C] per CTA, the
// row-major contract of mmo::host_srgemm (escalab/SIMD2 kernel/host_srgemm.h:17-49).
//
//   * Thread 0 issues 2D TMA loads (no multicast) of an A tile [BM rows][BK k]
//     (128-byte swizzle) and a B' tile into a STAGES-deep ring in shared
//     memory, with full/empty mbarriers per stage: the first STAGES tiles up
//     front, then each refill one tile after its stage is released.  (A
//     dedicated producer warp would put three warps on one SM sub-partition
//     and cap every thread at 168 registers.)
//   * B' is B with consecutive k rows interleaved in pairs,
//     B'[p][2j+e] = B[2p+e][j], written once per call by interleave_pairs
//     (prep.cu).  A thread then holds (A[i][2p], A[i][2p+1]) and
//     (B[2p][j], B[2p+1][j]) as register pairs, forms both products with one
//     packed f32x2 add/mul (each element rounded exactly like the scalar op),
//     and folds both into the accumulator with one three-operand min/max.
//   * 16 warps (4 per SM sub-partition); warp w owns rows {ty+16i} of the
//     column half 64*(w/8); each thread holds an 8 x 4 register tile (rows
//     ty+16i, columns 64*(w/8) + 32c + 2tx + e).  The tile is dispatch-bound:
//     the packed add and the three-operand min each occupy a 16-lane pipe for
//     two cycles per warp, i.e. one (x),(+) pair per lane per cycle.
//   * The epilogue applies (+) C, writes D with coalesced 8-byte stores and,
//     for the closure, sets one change flag per warp (warp vote + atomicOr).
//
// Out-of-range k is filled with NaN for the min/max semirings (TMA OOB fill
// for A, explicit padding for B'): a NaN product is dropped by min/max, so the
// tail adds nothing.  The summing semirings use zero fill.
#pragma once
#include "common.cuh"

namespace simd2 {

constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kBK = 32;
constexpr int kSimtWarps = 16;
constexpr int kSimtThreads = kSimtWarps * 32;
constexpr int kATileBytes = kBM * kBK * 4;  // 16 KiB
constexpr int kBTileBytes = kBK * kBN * 4;  // 16 KiB
constexpr int kStageBytes = kATileBytes + kBTileBytes;
constexpr int kSimtStages = 6;

constexpr size_t simt_smem_bytes(int stages) {
  return (size_t)stages * kStageBytes + 1024 /* alignment slack */ + 2 * stages * sizeof(uint64_t);
}

// Fused multiply-accumulate of two k terms into one output.
template <int OP>
struct Mac {
  __device__ static float mac2(float acc, float2 a, float2 b) {
    const float2 p = Semiring<OP>::mul2(a, b);
    return Semiring<OP>::add3(acc, p.x, p.y);
  }
  __device__ static float identity() { return Semiring<OP>::identity(); }
  __device__ static float add(float acc, float p) { return Semiring<OP>::add(acc, p); }
};

// plus_mul on CUDA cores (reference-precision FP32 path).
template <>
struct Mac<SIMD2_PLUS_MUL> {
  __device__ static float mac2(float acc, float2 a, float2 b) { return fmaf(a.y, b.y, fmaf(a.x, b.x, acc)); }
  __device__ static float identity() { return 0.0f; }
  __device__ static float add(float acc, float p) { return __fadd_rn(acc, p); }
};

// minus_square on CUDA cores: sum_k (a-b)^2.
template <>
struct Mac<SIMD2_MINUS_SQUARE> {
  __device__ static float mac2(float acc, float2 a, float2 b) {
    const float2 d = __fadd2_rn(a, make_float2(-b.x, -b.y));
    return fmaf(d.y, d.y, fmaf(d.x, d.x, acc));
  }
  __device__ static float identity() { return 0.0f; }
  __device__ static float add(float acc, float p) { return __fadd_rn(acc, p); }
};

struct EpilogueArgs {
  const float* C;
  long long ldc;
  float* D;
  long long ldd;
  int do_epilogue;
  int vec2;       // C/D rows are 8-byte aligned: use float2 accesses
  int* changed;   // nullable: set to 1 when any D element differs from C
  int conv_mode;  // simd2_conv, used with `changed`
  const int* gate;  // nullable: when *gate == 0 the kernel does nothing (closure
                    // step enqueued after the fixed point was reached)
  const int* gate2;  // nullable second gate (the FP16 / FP32 path choice)
  // Closure delta steps (square M = N = K, srgemm_simt_kernel only): chgA /
  // chgB, when set, receive a 1 for every 32 x 32 block of D that differs from
  // C, in the layouts of the occupancy maps (chgA[tile row][k-tile] for the
  // block's rows as an A block, chgB[k-tile][tile column] as a B block); dA /
  // dB, when set, are the previous step's maps, and a SKIP kernel keeps only
  // the k-tiles whose A or B block changed in that step.
  uint8_t* chgA;
  uint8_t* chgB;
  const uint8_t* dA;
  const uint8_t* dB;
};

__device__ __forceinline__ bool conv_changed(int mode, float old_v, float new_v) {
  if (mode == SIMD2_CONV_TOL) return fabsf(old_v - new_v) > 0.0001f;
  return __float_as_uint(old_v) != __float_as_uint(new_v);
}

template <int OP>
__device__ __forceinline__ float epilogue_value(int do_epi, int conv_mode, bool track, float v, float c,
                                                int& changed) {
  if (do_epi) v = Mac<OP>::add(v, c);
  if (conv_mode == SIMD2_CONV_APLP && v > -1.0f && v < 1.0f) v = -3.402823466e+38f;
  if (track && conv_changed(conv_mode, c, v)) changed = 1;
  return v;
}

// Largest k-tile count for which a skip list fits in shared memory.
constexpr int kMaxSkipKtiles = 4096;

// Distributed shared memory helpers (thread-block clusters).
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ float ld_dsmem_f32(const float* local_ptr, uint32_t rank) {
  uint32_t remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local_ptr)), "r"(rank));
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(remote) : "memory");
  return v;
}

// One CTA (or one CTA of a SPLIT-wide cluster) per 128 x 128 output tile.
//   SPLIT > 1 : the cluster's CTAs take every SPLIT-th k-tile of the tile's
//               k list, park their partial tile in shared memory, and each
//               CTA then folds 128/SPLIT rows of all partials (read through
//               distributed shared memory) with (+) and runs the epilogue on
//               them.  min/max are associative, so the result is exact.
//   SKIP      : the k list holds only the k-tiles whose A block (128 rows x
//               32 k) and B block (32 k x 128 columns) both contain an entry
//               other than the (x)-annihilator (occupancy maps occA, occB);
//               a skipped block can only produce identity products.  With
//               ep.dA / ep.dB (a closure step X_{t+1} = X_t (+) X_t (x) X_t
//               whose C is X_t) it also needs the A or the B block to have
//               changed in step t: every product of unchanged blocks was a
//               product of step t too and is already folded into X_t, so with
//               a min / max (+) it cannot change the result.
template <int OP, int STAGES, int SPLIT, bool SKIP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    srgemm_simt_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M,
                       int N, int K, EpilogueArgs ep, int tiles_m, int tiles_n, const uint8_t* __restrict__ occA,
                       const uint8_t* __restrict__ occB) {
  // A closure step enqueued after the previous step reported no change does
  // nothing; every CTA (every cluster member) sees the same word.
  if ((ep.gate && *ep.gate == 0) || (ep.gate2 && *ep.gate2 == 0)) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;
  __shared__ uint16_t s_klist[SKIP ? kMaxSkipKtiles : 1];
  __shared__ int s_warp_cnt[kSimtWarps];

  // Grouped raster: 8 consecutive tile rows share each B' column panel in L2.
  const int tile = blockIdx.x / SPLIT;
  const int rank = SPLIT > 1 ? (int)cluster_ctarank() : 0;
  const int group = 8;
  const int per_group = group * tiles_n;
  const int g = tile / per_group;
  const int first_m = g * group;
  const int gsize = min(tiles_m - first_m, group);
  const int local = tile - g * per_group;
  const int tm = first_m + local % gsize;
  const int tn = local / gsize;
  const int m0 = tm * kBM;
  const int n0 = tn * kBN;
  const int ktiles = (K + kBK - 1) / kBK;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kSimtWarps);
    }
    fence_mbar_init();
  }

  // ---- this CTA's k list: the tile's (occupied) k-tiles, every SPLIT-th one ----
  int nlist = ktiles;
  if constexpr (SKIP) {
    int running = 0;
    for (int base = 0; base < ktiles; base += kSimtThreads) {
      const int kt = base + threadIdx.x;
      const bool f = kt < ktiles && occA[(long long)tm * ktiles + kt] && occB[(long long)kt * tiles_n + tn] &&
                     (!ep.dA || ep.dA[(long long)tm * ktiles + kt] || ep.dB[(long long)kt * tiles_n + tn]);
      const unsigned ballot = __ballot_sync(0xffffffffu, f);
      if (lane == 0) s_warp_cnt[warp] = __popc(ballot);
      __syncthreads();
      int off = 0, total = 0;
      for (int w = 0; w < kSimtWarps; w++) {
        const int c = s_warp_cnt[w];
        off += w < warp ? c : 0;
        total += c;
      }
      if (f) s_klist[running + off + __popc(ballot & ((1u << lane) - 1u))] = (uint16_t)kt;
      running += total;
      __syncthreads();
    }
    nlist = running;
  }
  __syncthreads();
  // entries i = rank, rank + SPLIT, ... of the list
  const int nmine = nlist > rank ? (nlist - rank + SPLIT - 1) / SPLIT : 0;
  auto kt_of = [&](int i) -> int {
    const int li = rank + i * SPLIT;
    if constexpr (SKIP) return s_klist[li];
    else return li;
  };

  // Thread 0 issues the first STAGES k-tiles; refills happen inside the k loop.
  if (threadIdx.x == 0) {
    prefetch_tensormap(&tmA);
    prefetch_tensormap(&tmB);
    for (int i = 0; i < min(STAGES, nmine); i++) {
      const int kt = kt_of(i);
      uint8_t* sa = smem + i * kStageBytes;
      mbar_arrive_expect_tx(&full[i], kStageBytes);
      tma_load_2d(sa, &tmA, &full[i], kt * kBK, m0);
      tma_load_2d(sa + kATileBytes, &tmB, &full[i], 2 * n0, kt * (kBK / 2));
    }
  }

  constexpr int WN = 2;  // column pairs per thread
  const int tx = lane & 15;
  const int ty = (warp & 7) * 2 + (lane >> 4);
  const int cbase = (warp >> 3) * 64;
  const int swz = ty & 7;  // row & 7 for every row this thread reads (rows ty + 16 i)

  float acc[8][2 * WN];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 2 * WN; j++) acc[i][j] = Mac<OP>::identity();

  bool ok = true;
  int issued = min(STAGES, nmine);
  for (int i = 0; i < nmine; i++) {
    const int s = i % STAGES;
    // Refill the stage that list entry i-1 used once every warp has released it.
    if (threadIdx.x == 0 && i >= 1 && i - 1 + STAGES < nmine) {
      const int r = i - 1, rs = r % STAGES;
      if (mbar_wait(&empty[rs], (r / STAGES) & 1)) {
        uint8_t* sa = smem + rs * kStageBytes;
        const int nk = kt_of(r + STAGES);
        mbar_arrive_expect_tx(&full[rs], kStageBytes);
        tma_load_2d(sa, &tmA, &full[rs], nk * kBK, m0);
        tma_load_2d(sa + kATileBytes, &tmB, &full[rs], 2 * n0, nk * (kBK / 2));
        issued = r + STAGES + 1;
      } else {
        report_timeout(1);
      }
    }
    if (!mbar_wait(&full[s], (i / STAGES) & 1)) {
      report_timeout(2);
      ok = false;
      break;
    }
    const float* As = reinterpret_cast<const float*>(smem + s * kStageBytes);
    const float* Bs = reinterpret_cast<const float*>(smem + s * kStageBytes + kATileBytes);
#pragma unroll 2
    for (int q = 0; q < kBK / 4; q++) {
      float4 a[8];
#pragma unroll
      for (int ii = 0; ii < 8; ii++)
        a[ii] = *reinterpret_cast<const float4*>(As + (ty + 16 * ii) * kBK + ((q ^ swz) << 2));
#pragma unroll
      for (int h = 0; h < 2; h++) {
        float4 b[WN];
#pragma unroll
        for (int c = 0; c < WN; c++)
          b[c] = *reinterpret_cast<const float4*>(Bs + (2 * q + h) * (2 * kBN) + (cbase + 32 * c + 2 * tx) * 2);
#pragma unroll
        for (int ii = 0; ii < 8; ii++) {
          const float2 ap = h == 0 ? make_float2(a[ii].x, a[ii].y) : make_float2(a[ii].z, a[ii].w);
#pragma unroll
          for (int c = 0; c < WN; c++) {
            acc[ii][2 * c] = Mac<OP>::mac2(acc[ii][2 * c], ap, make_float2(b[c].x, b[c].y));
            acc[ii][2 * c + 1] = Mac<OP>::mac2(acc[ii][2 * c + 1], ap, make_float2(b[c].z, b[c].w));
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) {
    // Every issued copy must land before this CTA's shared memory is released.
    if (threadIdx.x == 0)
      for (int i = max(0, issued - STAGES); i < issued; i++) mbar_wait(&full[i % STAGES], (i / STAGES) & 1);
    if constexpr (SPLIT == 1) return;
  }

  // ---------------- epilogue ----------------
  const int do_epi = ep.do_epilogue;
  const int conv_mode = ep.conv_mode;
  const bool track = ep.changed != nullptr;
  const float* Cbase = ep.C;
  float* Dbase = ep.D;
  const long long ldc = ep.ldc, ldd = ep.ldd;
  int changed = 0;
  // bit 4 g + c: an element of the tile's 32 x 32 block (row group g, column
  // group c) changed (used only when ep.chgA is set)
  uint32_t bmask = 0;

  if constexpr (SPLIT == 1) {
    const int vec2 = ep.vec2;
    // The thread's C pairs are loaded first, all in flight together (each
    // load-then-use pair in turn would wait out the memory latency 16 times).
    float2 cpre[8][WN];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int row = m0 + ty + 16 * i;
#pragma unroll
      for (int c = 0; c < WN; c++) {
        const int col = n0 + cbase + 32 * c + 2 * tx;
        cpre[i][c] = (do_epi && vec2 && row < M && col + 1 < N)
                         ? *reinterpret_cast<const float2*>(Cbase + (long long)row * ldc + col)
                         : make_float2(0.f, 0.f);
      }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int row = m0 + ty + 16 * i;
      if (row < M) {
        const float* crow = Cbase + (long long)row * ldc;
        float* drow = Dbase + (long long)row * ldd;
#pragma unroll
        for (int c = 0; c < WN; c++) {
          const int col = n0 + cbase + 32 * c + 2 * tx;
          int ch = 0;
          if (vec2 && col + 1 < N) {
            const float2 cv = cpre[i][c];
            float2 v;
            v.x = epilogue_value<OP>(do_epi, conv_mode, track, acc[i][2 * c], cv.x, ch);
            v.y = epilogue_value<OP>(do_epi, conv_mode, track, acc[i][2 * c + 1], cv.y, ch);
            *reinterpret_cast<float2*>(drow + col) = v;
          } else {
#pragma unroll
            for (int e = 0; e < 2; e++) {
              if (col + e < N) {
                const float cv = do_epi ? crow[col + e] : 0.0f;
                drow[col + e] = epilogue_value<OP>(do_epi, conv_mode, track, acc[i][2 * c + e], cv, ch);
              }
            }
          }
          if (ch) {
            changed = 1;
            bmask |= 1u << (((i >> 1) << 2) | ((cbase >> 5) + c));  // row ty + 16 i lies in group i / 2
          }
        }
      }
    }
  } else {
    // Park the partial tile (row-major 128 x 128, padded rows) in the now idle stage memory.
    constexpr int kPitch = kBN + 4;
    float* part = reinterpret_cast<float*>(smem);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int c = 0; c < WN; c++) {
        const int r = ty + 16 * i, col = cbase + 32 * c + 2 * tx;
        part[r * kPitch + col] = acc[i][2 * c];
        part[r * kPitch + col + 1] = acc[i][2 * c + 1];
      }
    cluster_sync_all();  // every partial is in place
    constexpr int kRows = kBM / SPLIT;
    for (int e = threadIdx.x; e < kRows * kBN; e += kSimtThreads) {
      const int r = rank * kRows + e / kBN;
      const int col = e % kBN;
      float v = part[r * kPitch + col];
#pragma unroll
      for (int peer = 0; peer < SPLIT; peer++)
        if (peer != rank) v = Mac<OP>::add(v, ld_dsmem_f32(part + r * kPitch + col, (uint32_t)peer));
      const int row = m0 + r, gcol = n0 + col;
      if (ok && row < M && gcol < N) {
        const float cv = do_epi ? Cbase[(long long)row * ldc + gcol] : 0.0f;
        int ch = 0;
        Dbase[(long long)row * ldd + gcol] = epilogue_value<OP>(do_epi, conv_mode, track, v, cv, ch);
        if (ch) {
          changed = 1;
          bmask |= 1u << (((r >> 5) << 2) | (col >> 5));
        }
      }
    }
    cluster_sync_all();  // peers stay resident until every CTA has read their partials
  }
  if (track) {
    if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(ep.changed, 1);
  }
  if (ep.chgA) {
    // every writer stores 1, so no atomics; a set bit implies an element
    // inside the matrix, so both indices are in range
    const uint32_t m = __reduce_or_sync(0xffffffffu, bmask);
    if (lane == 0 && m) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (m & (0x1111u << q)) ep.chgA[(long long)tm * ktiles + 4 * tn + q] = 1;  // column group q
        if (m & (0xfu << (4 * q))) ep.chgB[(long long)(4 * tm + q) * tiles_n + tn] = 1;  // row group q
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FP16 selection kernel for max_min / min_max.  Used when every entry of A and
// B is exactly an FP16 value: (x) and (+) only select, so every product and
// every accumulator value is one of those FP16 values and the result is
// bit-identical to the FP32 computation.  Packed min/max.f16x2 handle two k
// values per lane per instruction (2 ALU instructions per 2 pairs instead of
// 3).  A is half [M][Kp] (128-byte swizzled TMA tiles of 128 rows x 64 k),
// B is k-pair words [Kp/2][Np] (tiles of 32 pair-rows x 128 words); the
// two halves of each accumulator hold the even- and odd-k partial results.
// ---------------------------------------------------------------------------
constexpr int kH2BK = 64;  // k per stage

__device__ __forceinline__ uint32_t hmin2u(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("min.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t hmax2u(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}

template <int OP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    srgemm_h2_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                     int K, EpilogueArgs ep, int tiles_m, int tiles_n) {
  static_assert(OP == SIMD2_MAX_MIN || OP == SIMD2_MIN_MAX, "selection semirings only");
  constexpr int STAGES = kSimtStages;
  if ((ep.gate && *ep.gate == 0) || (ep.gate2 && *ep.gate2 == 0)) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;

  const int group = 8;
  const int per_group = group * tiles_n;
  const int g = blockIdx.x / per_group;
  const int first_m = g * group;
  const int gsize = min(tiles_m - first_m, group);
  const int local = blockIdx.x - g * per_group;
  const int m0 = (first_m + local % gsize) * kBM;
  const int n0 = (local / gsize) * kBN;
  const int ktiles = (K + kH2BK - 1) / kH2BK;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kSimtWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    prefetch_tensormap(&tmA);
    prefetch_tensormap(&tmB);
    for (int kt = 0; kt < min(STAGES, ktiles); kt++) {
      uint8_t* sa = smem + kt * kStageBytes;
      mbar_arrive_expect_tx(&full[kt], kStageBytes);
      tma_load_2d(sa, &tmA, &full[kt], kt * kH2BK, m0);
      tma_load_2d(sa + kATileBytes, &tmB, &full[kt], n0, kt * (kH2BK / 2));
    }
  }

  const int tx = lane & 15;
  const int ty = (warp & 7) * 2 + (lane >> 4);
  const int cbase = (warp >> 3) * 64;
  const int swz = ty & 7;
  // identity of (+) in both halves: -inf (max) or +inf (min)
  const uint32_t ident = OP == SIMD2_MAX_MIN ? 0xfc00fc00u : 0x7c007c00u;
  uint32_t acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = ident;

  bool ok = true;
  int issued = min(STAGES, ktiles);
  for (int kt = 0; kt < ktiles; kt++) {
    const int s = kt % STAGES;
    if (threadIdx.x == 0 && kt >= 1 && kt - 1 + STAGES < ktiles) {
      const int r = kt - 1, rs = r % STAGES;
      if (mbar_wait(&empty[rs], (r / STAGES) & 1)) {
        uint8_t* sa = smem + rs * kStageBytes;
        const int nk = r + STAGES;
        mbar_arrive_expect_tx(&full[rs], kStageBytes);
        tma_load_2d(sa, &tmA, &full[rs], nk * kH2BK, m0);
        tma_load_2d(sa + kATileBytes, &tmB, &full[rs], n0, nk * (kH2BK / 2));
        issued = nk + 1;
      } else {
        report_timeout(3);
      }
    }
    if (!mbar_wait(&full[s], (kt / STAGES) & 1)) {
      report_timeout(4);
      ok = false;
      break;
    }
    const uint8_t* As = smem + s * kStageBytes;                               // 128 rows x 128 bytes
    const uint32_t* Bs = reinterpret_cast<const uint32_t*>(As + kATileBytes);  // 32 rows x 128 words
#pragma unroll 2
    for (int q = 0; q < 8; q++) {  // 16-byte chunk q = k pairs 4q .. 4q+3
      uint4 a[8];
#pragma unroll
      for (int i = 0; i < 8; i++)
        a[i] = *reinterpret_cast<const uint4*>(As + (ty + 16 * i) * 128 + ((q ^ swz) << 4));
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const int pr = 4 * q + h;
        uint2 b[2];
#pragma unroll
        for (int c = 0; c < 2; c++) b[c] = *reinterpret_cast<const uint2*>(Bs + pr * kBN + cbase + 32 * c + 2 * tx);
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const uint32_t ap = h == 0 ? a[i].x : h == 1 ? a[i].y : h == 2 ? a[i].z : a[i].w;
#pragma unroll
          for (int c = 0; c < 2; c++) {
            if constexpr (OP == SIMD2_MAX_MIN) {
              acc[i][2 * c] = hmax2u(acc[i][2 * c], hmin2u(ap, b[c].x));
              acc[i][2 * c + 1] = hmax2u(acc[i][2 * c + 1], hmin2u(ap, b[c].y));
            } else {
              acc[i][2 * c] = hmin2u(acc[i][2 * c], hmax2u(ap, b[c].x));
              acc[i][2 * c + 1] = hmin2u(acc[i][2 * c + 1], hmax2u(ap, b[c].y));
            }
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) {
    if (threadIdx.x == 0)
      for (int kt = max(0, issued - STAGES); kt < issued; kt++) mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1);
    return;
  }

  const int do_epi = ep.do_epilogue;
  const int conv_mode = ep.conv_mode;
  const bool track = ep.changed != nullptr;
  int changed = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int row = m0 + ty + 16 * i;
    if (row < M) {
      const float* crow = ep.C + (long long)row * ep.ldc;
      float* drow = ep.D + (long long)row * ep.ldd;
#pragma unroll
      for (int c = 0; c < 2; c++) {
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int col = n0 + cbase + 32 * c + 2 * tx + e;
          if (col < N) {
            const uint32_t w = acc[i][2 * c + e];
            const float lo = __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
            const float hi = __half2float(__ushort_as_half((unsigned short)(w >> 16)));
            const float v = Semiring<OP>::add(lo, hi);
            const float cv = do_epi ? crow[col] : 0.0f;
            drow[col] = epilogue_value<OP>(do_epi, conv_mode, track, v, cv, changed);
          }
        }
      }
    }
  }
  if (track) {
    if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(ep.changed, 1);
  }
}

// Block occupancy of X (rows x cols) in wide strips, optionally with entry
// counts.  A CTA of 256 threads covers 128 rows x 512 columns: warp w reads
// rows w, w + 8, ..., w + 120 and, per 128-column segment, each lane four
// consecutive columns (one 16-byte load when X's rows allow it), so every
// thread keeps 64 loads in flight.  occ32[bi][bj] = 1 when the 32 x 32 block
// holds an entry that is neither NaN nor `annihilator`.  With COUNTS,
// rowcnt[r] and colcnt[c] receive the entries that differ bitwise from the add
// identity `ident` (the entries a CSR copy of X stores): one atomic add per row
// and 512 columns, and per column and 128 rows (both zeroed before).
constexpr int kOccRows = 128;
constexpr int kOccCols = 512;

template <bool COUNTS>
__global__ void __launch_bounds__(256) occupancy_strip_kernel(const float* __restrict__ X, long long ldx, int rows,
                                                             int cols, float annihilator, float ident,
                                                             uint8_t* __restrict__ occ32, int bcols,
                                                             int* __restrict__ rowcnt, int* __restrict__ colcnt) {
  __shared__ int s_occ[kOccRows / 32][kOccCols / 32];
  __shared__ int s_col[COUNTS ? kOccCols : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = blockIdx.y * kOccRows, c0 = blockIdx.x * kOccCols;
  for (int i = threadIdx.x; i < (kOccRows / 32) * (kOccCols / 32); i += 256) (&s_occ[0][0])[i] = 0;
  if (COUNTS)
    for (int i = threadIdx.x; i < kOccCols; i += 256) s_col[i] = 0;
  __syncthreads();
  const bool vec = (ldx % 4 == 0) && (reinterpret_cast<uintptr_t>(X) % 16 == 0);
  const uint32_t id = __float_as_uint(ident);
  uint32_t flags = 0;  // bit rb * 4 + seg: an occupied entry in row block rb, segment seg
  int ccount[16];      // per segment seg, column e: entries of column c0 + 128 seg + 4 lane + e
#pragma unroll
  for (int i = 0; i < 16; i++) ccount[i] = 0;
  for (int rr = warp; rr < kOccRows; rr += 8) {
    const int r = r0 + rr;
    if (r >= rows) break;
    const float* xr = X + (long long)r * ldx;
    int rcount = 0;
#pragma unroll
    for (int seg = 0; seg < 4; seg++) {
      const int c = c0 + seg * 128 + lane * 4;
      float v[4];
      bool in[4];
      if (vec && c + 3 < cols) {
        const float4 u = __ldg(reinterpret_cast<const float4*>(xr + c));
        v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
#pragma unroll
        for (int e = 0; e < 4; e++) in[e] = true;
      } else {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          in[e] = c + e < cols;
          v[e] = in[e] ? __ldg(xr + c + e) : annihilator;
        }
      }
      bool f = false;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        f |= in[e] && (v[e] == v[e]) && (v[e] != annihilator);
        if (COUNTS) {
          const int st = in[e] && __float_as_uint(v[e]) != id;
          rcount += st;
          ccount[seg * 4 + e] += st;
        }
      }
      if (f) flags |= 1u << ((rr >> 5) * 4 + seg);
    }
    if (COUNTS) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) rcount += __shfl_xor_sync(0xffffffffu, rcount, o);
      if (lane == 0 && rcount) atomicAdd(&rowcnt[r], rcount);
    }
  }
  // a lane's four columns of segment seg lie in column block 4 seg + lane / 8
  for (uint32_t m = flags; m; m &= m - 1) {
    const int b = __ffs(m) - 1;
    atomicOr(&s_occ[b >> 2][(b & 3) * 4 + (lane >> 3)], 1);
  }
  if (COUNTS) {
#pragma unroll
    for (int i = 0; i < 16; i++)
      if (ccount[i]) atomicAdd(&s_col[(i >> 2) * 128 + lane * 4 + (i & 3)], ccount[i]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (kOccRows / 32) * (kOccCols / 32); i += 256) {
    const int bi = blockIdx.y * (kOccRows / 32) + i / (kOccCols / 32);
    const int bj = blockIdx.x * (kOccCols / 32) + i % (kOccCols / 32);
    if (bi * 32 < rows && bj * 32 < cols) occ32[(long long)bi * bcols + bj] = (uint8_t)(&s_occ[0][0])[i];
  }
  if (COUNTS)
    for (int i = threadIdx.x; i < kOccCols; i += 256)
      if (s_col[i] && c0 + i < cols) atomicAdd(&colcnt[c0 + i], s_col[i]);
}

// occ32[r / 32][c / 32] = 1 for every stored entry (r, c) of a CSR matrix
// (occ32 zeroed before); one warp per row.
__global__ void csr_occupancy32_kernel(int n, const int* __restrict__ rp, const int* __restrict__ cj,
                                       uint8_t* __restrict__ occ32, int bcols) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
    uint8_t* row = occ32 + (long long)(r >> 5) * bcols;
    for (int e = rp[r] + lane; e < rp[r + 1]; e += 32) {
      const int c = cj[e];
      if ((unsigned)c < (unsigned)n) row[c >> 5] = 1;
    }
  }
}

// stats[3] = sum_r rowcnt[r] (stored entries), stats[4] = sum_k rowcnt[k] *
// colcnt[k] (the products a Gustavson X (x) X forms); both zeroed before.
__global__ void count_products_kernel(int n, const int* __restrict__ rowcnt, const int* __restrict__ colcnt,
                                      unsigned long long* __restrict__ stats) {
  unsigned long long s = 0, p = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    s += (unsigned long long)rowcnt[k];
    p += (unsigned long long)rowcnt[k] * (unsigned long long)colcnt[k];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    p += __shfl_xor_sync(0xffffffffu, p, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s) atomicAdd(&stats[3], s);
    if (p) atomicAdd(&stats[4], p);
  }
}

// occA[tm][kt] = OR of occ32 over rows 4tm..4tm+3 at column block kt;
// occB[kt][tn] = OR of occ32 over row block kt, column blocks 4tn..4tn+3.
// Also counts surviving (tm, tn, kt) triples into stats[0], occupied A blocks
// into stats[1] and occupied B blocks into stats[2].
__global__ void occupancy_panels_kernel(const uint8_t* __restrict__ occ32A, int bcolsA, int browsA,
                                        const uint8_t* __restrict__ occ32B, int bcolsB, int browsB, int tiles_m,
                                        int tiles_n, int ktiles, uint8_t* __restrict__ occA,
                                        uint8_t* __restrict__ occB, unsigned long long* stats) {
  for (int kt = blockIdx.x; kt < ktiles; kt += gridDim.x) {
    __shared__ int s_ca, s_cb;
    if (threadIdx.x == 0) s_ca = s_cb = 0;
    __syncthreads();
    for (int tm = threadIdx.x; tm < tiles_m; tm += blockDim.x) {
      uint8_t v = 0;
      for (int q = 0; q < 4; q++) {
        const int bi = tm * 4 + q;
        if (bi < browsA && kt < bcolsA) v |= occ32A[(long long)bi * bcolsA + kt];
      }
      occA[(long long)tm * ktiles + kt] = v;
      if (v) atomicAdd(&s_ca, 1);
    }
    for (int tn = threadIdx.x; tn < tiles_n; tn += blockDim.x) {
      uint8_t v = 0;
      for (int q = 0; q < 4; q++) {
        const int bj = tn * 4 + q;
        if (kt < browsB && bj < bcolsB) v |= occ32B[(long long)kt * bcolsB + bj];
      }
      occB[(long long)kt * tiles_n + tn] = v;
      if (v) atomicAdd(&s_cb, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      atomicAdd(&stats[0], (unsigned long long)s_ca * (unsigned long long)s_cb);
      atomicAdd(&stats[1], (unsigned long long)s_ca);
      atomicAdd(&stats[2], (unsigned long long)s_cb);
    }
    __syncthreads();
  }
}

}  // namespace simd2
