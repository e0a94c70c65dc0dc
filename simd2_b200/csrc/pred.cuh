// pred.cuh -- closure with a predecessor matrix (path reconstruction).
//
// The Floyd-Warshall baselines of the reference keep, next to the distance
// matrix, pred[i][j] = the vertex before j on the best path found from i to
// j: i for an edge, -1 for no path and on the diagonal
// (apps/maxrp/baseline/main.cpp:80-94), and on a strict improvement through
// u, pred[i][j] = pred[u][j] (apps/maxrp/baseline/lib/apsp.cpp:19-22).
//
// Repeated squaring keeps the same invariant.  One step computes, per (i, j),
//   best = (+)_k X[i][k] (x) X[k][j]   over k = 0..n-1 in increasing order,
// with the host_srgemm accumulation (the running best is replaced only by a
// strictly better product, so the witness k* is the lowest k attaining it),
// then
//   X'[i][j] = best (+) X[i][j]                      (host_srgemm epilogue)
//   P'[i][j] = best strictly better than X[i][j] ? P[k*][j] : P[i][j]
// since j's predecessor on the path i -> k* -> j is its predecessor on k* -> j.
//
// pred_fast_kernel finds k* without a compare per product.  It runs the
// packed main loop of the CUDA-core srgemm tile (TMA-staged A and k-pair
// interleaved B', one (x),(+) pair per lane per cycle) into a per-k-tile
// minimum t, and after each k-tile of 32 keeps, per output, best and the index
// of the last k-tile where t was strictly better than best.  That k-tile holds
// k*: every earlier k-tile's products are worse than best (strict record), and
// no later one is better.  The epilogue re-forms the 32 products of that
// k-tile for each output whose value improves (X[i][k] from the row, X[k][j]
// from a transposed copy, both contiguous) and takes the first one equal to
// best -- the same IEEE operation on the same operands, so the same bits.
// The re-scan loads all 32 operand pairs before comparing (one memory round
// trip per output instead of up to 32 dependent ones).
#pragma once
#include "common.cuh"
#include "srgemm_simt.cuh"

namespace simd2 {

template <int OP>
struct PredOps;
// mul exactly as the oracle (host_srgemm functors); better(p, best) is the
// strict comparison of the add functor: minimum replaces on rhs < lhs,
// maximum on lhs < rhs.
template <>
struct PredOps<SIMD2_MIN_PLUS> {
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
  __device__ static bool better(float p, float best) { return p < best; }
  static constexpr bool kMin = true;
};
template <>
struct PredOps<SIMD2_MAX_PLUS> {
  __device__ static float mul(float a, float b) { return __fadd_rn(a, b); }
  __device__ static bool better(float p, float best) { return best < p; }
  static constexpr bool kMin = false;
};
template <>
struct PredOps<SIMD2_MAX_MIN> {
  __device__ static float mul(float a, float b) { return (b < a) ? b : a; }
  __device__ static bool better(float p, float best) { return best < p; }
  static constexpr bool kMin = false;
};
template <>
struct PredOps<SIMD2_MAX_MUL> {
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ static bool better(float p, float best) { return best < p; }
  static constexpr bool kMin = false;
};
template <>
struct PredOps<SIMD2_MIN_MUL> {
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ static bool better(float p, float best) { return p < best; }
  static constexpr bool kMin = true;
};
template <>
struct PredOps<SIMD2_MIN_MAX> {
  __device__ static float mul(float a, float b) { return (a < b) ? b : a; }
  __device__ static bool better(float p, float best) { return p < best; }
  static constexpr bool kMin = true;
};

// Row stride (uint16 entries) of the per-output k-tile record in shared
// memory; 160 puts the two half-warps' rows on different banks.
constexpr int kPredRecStride = 160;
constexpr int kPredStages = 4;

constexpr size_t pred_smem_bytes() {
  return simt_smem_bytes(kPredStages) + (size_t)kBM * kPredRecStride * sizeof(uint16_t);
}

// The lowest k in [k0, k0 + 32) with X[i][k] (x) X[k][j] == b, or -1; xr and
// tr point at X[i][k0] and X^T[j][k0].  All 32 operand pairs are loaded before
// the compares (16-byte loads when vec4 and the k-tile is whole), so an output
// costs one memory round trip.  One copy of the code for all call sites.
template <int OP>
__device__ __noinline__ int pred_witness(const float* __restrict__ xr, const float* __restrict__ tr, int k0, int n,
                                         float b, int vec4) {
  using O = PredOps<OP>;
  uint32_t hit = 0;
  if (vec4 && k0 + kBK <= n) {
#pragma unroll
    for (int q = 0; q < kBK / 4; q++) {
      const float4 x4 = __ldg(reinterpret_cast<const float4*>(xr) + q);
      const float4 t4 = __ldg(reinterpret_cast<const float4*>(tr) + q);
      hit |= ((uint32_t)(O::mul(x4.x, t4.x) == b) << (4 * q)) | ((uint32_t)(O::mul(x4.y, t4.y) == b) << (4 * q + 1)) |
             ((uint32_t)(O::mul(x4.z, t4.z) == b) << (4 * q + 2)) |
             ((uint32_t)(O::mul(x4.w, t4.w) == b) << (4 * q + 3));
    }
  } else {
#pragma unroll
    for (int kk = 0; kk < kBK; kk++)
      if (k0 + kk < n && O::mul(__ldg(xr + kk), __ldg(tr + kk)) == b) hit |= 1u << kk;
  }
  return hit ? k0 + __ffs(hit) - 1 : -1;
}

// One predecessor-tracking squaring step on a 128 x 128 output tile per CTA:
// X, P (pitch ldx, ldp) -> Xn, Pn (pitch ldxn, ldpn).  tmA reads X in k-tiles
// (NaN beyond n), tmB the k-pair interleaved copy of X, XT is X transposed
// (pitch ldt).  *changed |= 1 when any X' element differs bitwise from X.
template <int OP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    pred_fast_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int n,
                     const float* __restrict__ X, long long ldx, const float* __restrict__ XT, long long ldt,
                     const int32_t* __restrict__ P, long long ldp, float* __restrict__ Xn, long long ldxn,
                     int32_t* __restrict__ Pn, long long ldpn, int* __restrict__ changed, int tiles_m,
                     int tiles_n, int vec4) {
  using O = PredOps<OP>;
  constexpr int STAGES = kPredStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;
  uint16_t* rec = reinterpret_cast<uint16_t*>(empty + STAGES);

  // grouped raster: 8 consecutive tile rows share each B' column panel in L2
  const int tile = blockIdx.x;
  const int per_group = 8 * tiles_n;
  const int g = tile / per_group;
  const int first_m = g * 8;
  const int gsize = min(tiles_m - first_m, 8);
  const int local = tile - g * per_group;
  const int m0 = (first_m + local % gsize) * kBM;
  const int n0 = (local / gsize) * kBN;
  const int ktiles = (n + kBK - 1) / kBK;
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
    for (int i = 0; i < min(STAGES, ktiles); i++) {
      uint8_t* sa = smem + i * kStageBytes;
      mbar_arrive_expect_tx(&full[i], kStageBytes);
      tma_load_2d(sa, &tmA, &full[i], i * kBK, m0);
      tma_load_2d(sa + kATileBytes, &tmB, &full[i], 2 * n0, i * (kBK / 2));
    }
  }

  const int tx = lane & 15;
  const int ty = (warp & 7) * 2 + (lane >> 4);
  const int cbase = (warp >> 3) * 64;
  const int swz = ty & 7;
  const float ident = Mac<OP>::identity();
  float best[8][4], t[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) best[i][j] = ident;

  bool ok = true;
  int issued = min(STAGES, ktiles);
  for (int kt = 0; kt < ktiles; kt++) {
    const int s = kt % STAGES;
    if (threadIdx.x == 0 && kt >= 1 && kt - 1 + STAGES < ktiles) {
      const int r = kt - 1, rs = r % STAGES;
      if (mbar_wait(&empty[rs], (r / STAGES) & 1)) {
        uint8_t* sa = smem + rs * kStageBytes;
        mbar_arrive_expect_tx(&full[rs], kStageBytes);
        tma_load_2d(sa, &tmA, &full[rs], (r + STAGES) * kBK, m0);
        tma_load_2d(sa + kATileBytes, &tmB, &full[rs], 2 * n0, (r + STAGES) * (kBK / 2));
        issued = r + STAGES + 1;
      } else {
        report_timeout(21);
      }
    }
    if (!mbar_wait(&full[s], (kt / STAGES) & 1)) {
      report_timeout(22);
      ok = false;
      break;
    }
    const float* As = reinterpret_cast<const float*>(smem + s * kStageBytes);
    const float* Bs = reinterpret_cast<const float*>(smem + s * kStageBytes + kATileBytes);
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) t[i][j] = ident;
#pragma unroll 2
    for (int q = 0; q < kBK / 4; q++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        float2 a[8];
#pragma unroll
        for (int ii = 0; ii < 8; ii++)
          a[ii] = *reinterpret_cast<const float2*>(As + (ty + 16 * ii) * kBK + ((q ^ swz) << 2) + 2 * h);
        float4 b[2];
#pragma unroll
        for (int c = 0; c < 2; c++)
          b[c] = *reinterpret_cast<const float4*>(Bs + (2 * q + h) * (2 * kBN) + (cbase + 32 * c + 2 * tx) * 2);
#pragma unroll
        for (int ii = 0; ii < 8; ii++)
#pragma unroll
          for (int c = 0; c < 2; c++) {
            t[ii][2 * c] = Mac<OP>::mac2(t[ii][2 * c], a[ii], make_float2(b[c].x, b[c].y));
            t[ii][2 * c + 1] = Mac<OP>::mac2(t[ii][2 * c + 1], a[ii], make_float2(b[c].z, b[c].w));
          }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    // strict record: the k-tile where best last improved holds the witness
#pragma unroll
    for (int ii = 0; ii < 8; ii++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (O::better(t[ii][j], best[ii][j])) {
          best[ii][j] = t[ii][j];
          rec[(ty + 16 * ii) * kPredRecStride + cbase + 32 * (j >> 1) + 2 * tx + (j & 1)] = (uint16_t)kt;
        }
      }
  }
  if (!ok) {
    // every issued copy lands before this CTA's shared memory is released
    if (threadIdx.x == 0)
      for (int i = max(0, issued - STAGES); i < issued; i++) mbar_wait(&full[i % STAGES], (i / STAGES) & 1);
    return;
  }
  __syncwarp();

  int ch = 0;
#pragma unroll
  for (int ii = 0; ii < 8; ii++) {
    const int i = m0 + ty + 16 * ii;
    if (i >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int cl = cbase + 32 * (j >> 1) + 2 * tx + (j & 1);
      const int col = n0 + cl;
      if (col >= n) continue;
      const float cv = X[(long long)i * ldx + col];
      const float b = best[ii][j];
      // host_srgemm epilogue: D = addop(D, C) with D = best
      const float xn = O::kMin ? ((cv < b) ? cv : b) : ((b < cv) ? cv : b);
      int32_t pv;
      if (O::better(b, cv)) {
        const int k0 = (int)rec[(ty + 16 * ii) * kPredRecStride + cl] * kBK;
        int ks = pred_witness<OP>(X + (long long)i * ldx + k0, XT + (long long)col * ldt + k0, k0, n, b, vec4);
        if (ks < 0) {
          // cannot happen with the precondition (no NaN, no -0.0): the
          // product that set best is re-formed with the same operation
          report_error(SIMD2_ERR_INVALID_ARG);
          ks = i;
        }
        pv = P[(long long)ks * ldp + col];
      } else {
        pv = P[(long long)i * ldp + col];
      }
      Xn[(long long)i * ldxn + col] = xn;
      Pn[(long long)i * ldpn + col] = pv;
      if (__float_as_uint(xn) != __float_as_uint(cv)) ch = 1;
    }
  }
  if (__any_sync(0xffffffffu, ch) && lane == 0) atomicOr(changed, 1);
}

// XT[j][i] = X[i][j] for i, j < n, through 32 x 32 shared-memory tiles.
__global__ void transpose_f32_kernel(int n, const float* __restrict__ X, long long ldx, float* __restrict__ XT,
                                     long long ldt) {
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = by + r, j = bx + threadIdx.x;
    if (i < n && j < n) tile[r][threadIdx.x] = X[(long long)i * ldx + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = bx + r, i = by + threadIdx.x;
    if (i < n && j < n) XT[(long long)j * ldt + i] = tile[threadIdx.x][r];
  }
}
// P[i][j] = i where X[i][j] is an edge (not the add identity) and i != j, else -1.
__global__ void pred_init_kernel(int n, const float* __restrict__ X, long long ldx, int32_t* __restrict__ P,
                                 long long ldp, float ident) {
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    const float x = X[(long long)i * ldx + j];
    P[(long long)i * ldp + j] = (i != j && __float_as_uint(x) != __float_as_uint(ident)) ? i : -1;
  }
}

}  // namespace simd2
