// closure_batched.cuh -- many independent closures in one persistent launch.
//
// Each graph g (n_g vertices) is closed by repeated squaring X <- X (+) X(x)X
// until unchanged, as in the reference's closure apps
// (apps/apsp/cuASR/apsp_cuASR.cu:37-54, convergence kernel/converge.cuh:6-69).
// One CTA owns one graph at a time and runs its whole closure, so no CTA ever
// waits for another: graphs are taken from an atomic queue in descending size
// (longest-processing-time first) until the queue is empty.
//
// Per graph the workspace holds two ping-pong copies of X in the normal
// layout [Mp][Kp] and two in the k-pair interleaved layout X'[Kp/2][2Np]
// (the B operand of the CUDA-core micro-kernel, see srgemm_simt.cuh).  All
// padding (rows/cols >= n) is NaN, written once by the prep kernel and never
// overwritten, so every tile load is in bounds and a padded k contributes a
// NaN product, which min/max drop.  Tiles are staged by TMA through
// per-graph tensor maps kept in device memory (encoded once per plan) into
// the same kSimtStages-deep mbarrier ring as the single srgemm (the launch
// sizes shared memory from that same constant), with the barrier
// phases running on across tiles and graphs; the epilogue of iteration t
// writes both layouts of X_{t+1} and a per-graph change flag, then a
// generic-to-async proxy fence orders those writes before the next step's
// TMA reads.
#pragma once
#include "srgemm_simt.cuh"

namespace simd2 {

struct BatchGraph {
  int n;        // vertices
  int Mp;       // rows padded to a multiple of 128
  int Kp;       // columns (= k extent) padded to a multiple of 32
  int Np;       // columns padded to a multiple of 128 (interleaved layout)
  float* X[2];  // [Mp][Kp], ping-pong
  float* P[2];  // [Kp/2][2*Np] interleaved, ping-pong
  // FP16 copies for the selection semirings (max_min, min_max), else null:
  int Kh;           // columns (= k extent) padded to a multiple of 64
  __half* Xh[2];    // [Mp][Kh], ping-pong
  uint32_t* Ph[2];  // [Kh/2][Np] k-pair words (X[2p][j], X[2p+1][j]), ping-pong
  float* user;  // caller's matrix (result is copied back here)
  long long ldu;
  int iters;    // out: steps run (including the final unchanged one)
  int changed;  // out: 1 if the last step still changed something
};

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Tensor maps of one graph, in device memory: A role X[0], X[1] ([Mp][Kp],
// 128 x 32 boxes, 128-byte swizzle) and B role P[0], P[1] ([Kp/2][2Np],
// 16 x 256 boxes).  Encoded once on the host when the plan is made.
struct BatchMaps {
  CUtensorMap a[2];
  CUtensorMap b[2];
  CUtensorMap ah[2];  // Xh[0], Xh[1]: 128 rows x 64 halves, 128-byte swizzle (FP16 path)
  CUtensorMap bh[2];  // Ph[0], Ph[1]: 32 pair rows x 128 words (FP16 path)
};

// One k-tile of the 8 x 4 register tile; ROWS < 8 skips rows ty + 16i for
// i >= ROWS (tile rows 16 ROWS..127), used when those rows lie past the graph.
// Q = 8 runs the whole k-tile; Q = 0 runs its first qn groups of 4 k (the
// graph's last k-tile: groups wholly past column n hold only NaN padding,
// whose products min/max drop).
template <int OP, int ROWS, int Q>
__device__ __forceinline__ void batched_mac_ktile(float (&acc)[8][4], const float* As, const float* Bs, int ty,
                                                  int tx, int cbase, int swz, int qn) {
  constexpr int WN = 2;
  const int qe = Q ? Q : qn;
#pragma unroll 2
  for (int q = 0; q < qe; q++) {
    float4 a[ROWS];
#pragma unroll
    for (int ii = 0; ii < ROWS; ii++)
      a[ii] = *reinterpret_cast<const float4*>(As + (ty + 16 * ii) * kBK + ((q ^ swz) << 2));
#pragma unroll
    for (int h = 0; h < 2; h++) {
      float4 b[WN];
#pragma unroll
      for (int c = 0; c < WN; c++)
        b[c] = *reinterpret_cast<const float4*>(Bs + (2 * q + h) * (2 * kBN) + (cbase + 32 * c + 2 * tx) * 2);
#pragma unroll
      for (int ii = 0; ii < ROWS; ii++) {
        const float2 ap = h == 0 ? make_float2(a[ii].x, a[ii].y) : make_float2(a[ii].z, a[ii].w);
#pragma unroll
        for (int c = 0; c < WN; c++) {
          acc[ii][2 * c] = Mac<OP>::mac2(acc[ii][2 * c], ap, make_float2(b[c].x, b[c].y));
          acc[ii][2 * c + 1] = Mac<OP>::mac2(acc[ii][2 * c + 1], ap, make_float2(b[c].z, b[c].w));
        }
      }
    }
  }
}

template <int OP, int Q>
__device__ __forceinline__ void batched_mac_rows(int row_groups, float (&acc)[8][4], const float* As, const float* Bs,
                                                 int ty, int tx, int cbase, int swz, int qn) {
  switch (row_groups) {
    case 1: batched_mac_ktile<OP, 1, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 2: batched_mac_ktile<OP, 2, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 3: batched_mac_ktile<OP, 3, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 4: batched_mac_ktile<OP, 4, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 5: batched_mac_ktile<OP, 5, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 6: batched_mac_ktile<OP, 6, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 7: batched_mac_ktile<OP, 7, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    default: batched_mac_ktile<OP, 8, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
  }
}

template <int OP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    closure_batched_kernel(BatchGraph* graphs, const BatchMaps* __restrict__ maps, const int* order, int count,
                           int* queue, int max_iter, int conv_mode, const int* fp16_bad) {
  constexpr int STAGES = kSimtStages;
  // with the FP16 path enqueued too, this kernel runs only when some entry is not an FP16 value
  if (fp16_bad && *fp16_bad == 0) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;
  __shared__ int s_graph;
  __shared__ int s_changed;
  __shared__ int s_failed;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int tx = lane & 15;
  const int ty = (warp & 7) * 2 + (lane >> 4);
  const int cbase = (warp >> 3) * 64;
  const int swz = ty & 7;
  constexpr int WN = 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kSimtWarps);
    }
    fence_mbar_init();
    s_failed = 0;
  }
  __syncthreads();
  // Running k-tile counter of this CTA: load number g uses stage g % STAGES
  // with phase parity (g / STAGES) & 1, across tiles, iterations and graphs.
  uint32_t gk = 0;

  while (true) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(queue, 1);
      s_graph = (q < count && !s_failed) ? order[q] : -1;
    }
    __syncthreads();
    const int gi = s_graph;
    if (gi < 0) break;
    BatchGraph& G = graphs[gi];
    const BatchMaps* mp = maps + gi;
    const int n = G.n, Kp = G.Kp, Np = G.Np;
    const int tiles_m = G.Mp / kBM, tiles_n = Np / kBN, ktiles = Kp / kBK;
    int it = 0, changed_any = 1;
    while (changed_any && it < max_iter) {
      const int cur = it & 1, nxt = cur ^ 1;
      const float* X = G.X[cur];
      float* Xn = G.X[nxt];
      float* Pn = G.P[nxt];
      const CUtensorMap* tmA = &mp->a[cur];
      const CUtensorMap* tmB = &mp->b[cur];
      if (threadIdx.x == 0) s_changed = 0;
      __syncthreads();
      int changed = 0;
      // The step's loads form one stream over (tile, k): load j = tile j / ktiles,
      // k-tile j % ktiles, so the next tile's first loads are in flight while the
      // current tile runs its epilogue.
      const int ntiles = tiles_m * tiles_n;
      const int nloads = ntiles * ktiles;
      auto issue = [&](int j) {
        const uint32_t g = gk + j;
        const int s = g % STAGES;
        if (!mbar_wait(&empty[s], ((g / STAGES) & 1) ^ 1)) {
          report_timeout(21);
          s_failed = 1;
        }
        const int tile = j / ktiles, kk = j - tile * ktiles;
        uint8_t* sa = smem + s * kStageBytes;
        mbar_arrive_expect_tx(&full[s], kStageBytes);
        tma_load_2d(sa, tmA, &full[s], kk * kBK, (tile % tiles_m) * kBM);
        tma_load_2d(sa + kATileBytes, tmB, &full[s], 2 * (tile / tiles_m) * kBN, kk * (kBK / 2));
      };
      if (threadIdx.x == 0)
        for (int j = 0; j < min(STAGES, nloads); j++) issue(j);
      for (int t = 0; t < ntiles; t++) {
        const int m0 = (t % tiles_m) * kBM;
        const int n0 = (t / tiles_m) * kBN;
        const int row_groups = min(8, (n - m0 + 15) / 16);  // 16-row groups holding graph rows
        const bool idle_cols = n0 + 64 >= n && cbase == 64;  // uniform over the warp
        float acc[8][2 * WN];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int j = 0; j < 2 * WN; j++) acc[i][j] = Mac<OP>::identity();
        for (int i = 0; i < ktiles; i++) {
          const int j = t * ktiles + i;
          const uint32_t g = gk + j;
          const int s = g % STAGES;
          // refill: load j-1+STAGES goes into the stage that load j-1 used
          if (threadIdx.x == 0 && j >= 1 && j - 1 + STAGES < nloads) issue(j - 1 + STAGES);
          if (!mbar_wait(&full[s], (g / STAGES) & 1)) {
            report_timeout(23);
            s_failed = 1;
          }
          const float* As = reinterpret_cast<const float*>(smem + s * kStageBytes);
          const float* Bs = reinterpret_cast<const float*>(smem + s * kStageBytes + kATileBytes);
          // Padding: 16-row groups past the graph are not computed, and
          // the warps of the upper column half sit out a tile whose columns end
          // by column 64 -- what they would compute is never stored.
          if (!idle_cols) {
            // groups of 4 k of this k-tile that hold graph columns
            const int qn = min(kBK / 4, (n - i * kBK + 3) >> 2);
            if (qn == kBK / 4) batched_mac_rows<OP, kBK / 4>(row_groups, acc, As, Bs, ty, tx, cbase, swz, qn);
            else batched_mac_rows<OP, 0>(row_groups, acc, As, Bs, ty, tx, cbase, swz, qn);
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[s]);
        }
        // epilogue: X_{t+1} = X_t (+) acc in both layouts, change test against
        // X_t.  The thread's 32 old values are loaded first, as 8-byte pairs
        // (col is even and Kp a multiple of 32, so a pair starting below n
        // lies inside the padded row) all in flight together, then combined.
        float2 oldv[8][WN];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int row = m0 + ty + 16 * i;
#pragma unroll
          for (int c = 0; c < WN; c++) {
            const int col = n0 + cbase + 32 * c + 2 * tx;
            oldv[i][c] = (row < n && col < n)
                             ? __ldcg(reinterpret_cast<const float2*>(X + (long long)row * Kp + col))
                             : make_float2(0.f, 0.f);
          }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int row = m0 + ty + 16 * i;
          if (row < n) {
#pragma unroll
            for (int c = 0; c < WN; c++) {
              const int col = n0 + cbase + 32 * c + 2 * tx;
#pragma unroll
              for (int e = 0; e < 2; e++) {
                if (col + e < n) {
                  const float old_v = e == 0 ? oldv[i][c].x : oldv[i][c].y;
                  float v = Mac<OP>::add(acc[i][2 * c + e], old_v);
                  if (conv_mode == SIMD2_CONV_APLP && v > -1.0f && v < 1.0f) v = -3.402823466e+38f;
                  if (conv_changed(conv_mode, old_v, v)) changed = 1;
                  Xn[(long long)row * Kp + col + e] = v;
                  Pn[(long long)(row >> 1) * (2LL * Np) + 2 * (col + e) + (row & 1)] = v;
                }
              }
            }
          }
        }
      }
      gk += nloads;
      if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(&s_changed, 1);
      // X_{t+1} was written through the generic proxy; the next step reads it with TMA.
      fence_proxy_async_global();
      __syncthreads();
      changed_any = s_changed && !s_failed;
      it++;
    }
    if (threadIdx.x == 0) {
      G.iters = it;
      G.changed = changed_any || s_failed;
    }
    __syncthreads();
  }
}

// Prep: copy every graph into X[0] (normal) and P[0] (interleaved), NaN padding;
// X[1], P[1] get the same padding (their valid region is written by step 1).
// One CTA row per (graph, padded row); grid-stride over graphs.  With the
// FP16 path enqueued too, it runs only when some entry is not an FP16 value.
__global__ void batched_prep_kernel(BatchGraph* graphs, int count, const int* fp16_bad) {
  if (fp16_bad && *fp16_bad == 0) return;
  const float nanv = __int_as_float(0x7fc00000);
  for (int g = blockIdx.y; g < count; g += gridDim.y) {
    BatchGraph& G = graphs[g];
    const int n = G.n, Kp = G.Kp, Np = G.Np, Mp = G.Mp;
    // normal layout, both buffers
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)Mp * Kp;
         t += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(t / Kp), k = (int)(t - (long long)i * Kp);
      const float v = (i < n && k < n) ? G.user[(long long)i * G.ldu + k] : nanv;
      G.X[0][t] = v;
      G.X[1][t] = nanv;
    }
    // interleaved layout, both buffers: P[p][2j+e] = X[2p+e][j]
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)(Kp / 2) * 2 * Np;
         t += (long long)gridDim.x * blockDim.x) {
      const int p = (int)(t / (2LL * Np));
      const int r = (int)(t - (long long)p * 2 * Np);
      const int j = r >> 1, k = 2 * p + (r & 1);
      const float v = (k < n && j < n) ? G.user[(long long)k * G.ldu + j] : nanv;
      G.P[0][t] = v;
      G.P[1][t] = nanv;
    }
  }
}

// Copy every result X[iters & 1] (or its FP16 twin, when the FP16 path ran)
// back into the caller's matrix.
__global__ void batched_finish_kernel(BatchGraph* graphs, int count, const int* fp16_bad) {
  const bool h = fp16_bad && *fp16_bad == 0;
  for (int g = blockIdx.y; g < count; g += gridDim.y) {
    BatchGraph& G = graphs[g];
    const int n = G.n;
    if (h) {
      const __half* R = G.Xh[G.iters & 1];
      const int Kh = G.Kh;
      for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
           t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t - (long long)i * n);
        G.user[(long long)i * G.ldu + j] = __half2float(R[(long long)i * Kh + j]);
      }
    } else {
      const float* R = G.X[G.iters & 1];
      const int Kp = G.Kp;
      for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
           t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t - (long long)i * n);
        G.user[(long long)i * G.ldu + j] = R[(long long)i * Kp + j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FP16 path of the selection semirings (max_min, min_max).  Their closure only
// ever selects among the input entries (and the identities), so when every
// entry of every graph is exactly an FP16 value, every X_t is too, and the
// packed min/max.f16x2 micro-kernel of srgemm_h2_kernel (two k per lane per
// instruction: 2 ALU instructions per 2 (x),(+) pairs instead of 3) gives the
// FP32 closure's bits.  batched_prep_h_kernel writes the FP16 copies and sets
// *fp16_bad when an entry is not an FP16 value; the FP16 and FP32 closure
// kernels are both enqueued, each gated by that flag, so the plan's run stays
// asynchronous.
// ---------------------------------------------------------------------------
__device__ __forceinline__ __half batched_half_exact(float x, bool& bad) {
  const __half h = __float2half_rn(x);
  bad |= __float_as_uint(__half2float(h)) != __float_as_uint(x);
  return h;
}

// Xh[0] = X as halves [Mp][Kh], Ph[0] = k-pair words [Kh/2][Np], NaN padding;
// Xh[1], Ph[1] = NaN (their valid region is written by step 1).
__global__ void batched_prep_h_kernel(BatchGraph* graphs, int count, int* fp16_bad) {
  const __half nanh = __ushort_as_half(0x7e00);
  const uint32_t nanw = 0x7e007e00u;
  bool bad = false;
  for (int g = blockIdx.y; g < count; g += gridDim.y) {
    BatchGraph& G = graphs[g];
    const int n = G.n, Kh = G.Kh, Np = G.Np, Mp = G.Mp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)Mp * Kh;
         t += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(t / Kh), k = (int)(t - (long long)i * Kh);
      G.Xh[0][t] = (i < n && k < n) ? batched_half_exact(G.user[(long long)i * G.ldu + k], bad) : nanh;
      G.Xh[1][t] = nanh;
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)(Kh / 2) * Np;
         t += (long long)gridDim.x * blockDim.x) {
      const int p = (int)(t / Np), j = (int)(t - (long long)p * Np);
      const int k0 = 2 * p, k1 = 2 * p + 1;
      const __half lo = (k0 < n && j < n) ? batched_half_exact(G.user[(long long)k0 * G.ldu + j], bad) : nanh;
      const __half hi = (k1 < n && j < n) ? batched_half_exact(G.user[(long long)k1 * G.ldu + j], bad) : nanh;
      G.Ph[0][t] = (uint32_t)__half_as_ushort(lo) | ((uint32_t)__half_as_ushort(hi) << 16);
      G.Ph[1][t] = nanw;
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(fp16_bad, 1);
}

__device__ __forceinline__ uint32_t bh_min2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("min.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t bh_max2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}

// One 64-k tile of the FP16 8 x 4 register tile (rows ty + 16i, i < ROWS):
// A chunk q (k pairs 4q..4q+3 of a row, 16 bytes) sits at chunk q ^ (row & 7)
// of the 128-byte row; B pair row pr holds 128 words.  Q = 8: the whole
// k-tile; Q = 0: its first qn chunks of 8 k (the rest is NaN padding).
template <int OP, int ROWS, int Q>
__device__ __forceinline__ void batched_h2_ktile(uint32_t (&acc)[8][4], const uint8_t* As, const uint32_t* Bs, int ty,
                                                 int tx, int cbase, int swz, int qn) {
  const int qe = Q ? Q : qn;
#pragma unroll 2
  for (int q = 0; q < qe; q++) {
    uint4 a[ROWS];
#pragma unroll
    for (int i = 0; i < ROWS; i++) a[i] = *reinterpret_cast<const uint4*>(As + (ty + 16 * i) * 128 + ((q ^ swz) << 4));
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int pr = 4 * q + h;
      uint2 b[2];
#pragma unroll
      for (int c = 0; c < 2; c++) b[c] = *reinterpret_cast<const uint2*>(Bs + pr * kBN + cbase + 32 * c + 2 * tx);
#pragma unroll
      for (int i = 0; i < ROWS; i++) {
        const uint32_t ap = h == 0 ? a[i].x : h == 1 ? a[i].y : h == 2 ? a[i].z : a[i].w;
#pragma unroll
        for (int c = 0; c < 2; c++) {
          if constexpr (OP == SIMD2_MAX_MIN) {
            acc[i][2 * c] = bh_max2(acc[i][2 * c], bh_min2(ap, b[c].x));
            acc[i][2 * c + 1] = bh_max2(acc[i][2 * c + 1], bh_min2(ap, b[c].y));
          } else {
            acc[i][2 * c] = bh_min2(acc[i][2 * c], bh_max2(ap, b[c].x));
            acc[i][2 * c + 1] = bh_min2(acc[i][2 * c + 1], bh_max2(ap, b[c].y));
          }
        }
      }
    }
  }
}

template <int OP, int Q>
__device__ __forceinline__ void batched_h2_rows(int row_groups, uint32_t (&acc)[8][4], const uint8_t* As,
                                                const uint32_t* Bs, int ty, int tx, int cbase, int swz, int qn) {
  switch (row_groups) {
    case 1: batched_h2_ktile<OP, 1, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 2: batched_h2_ktile<OP, 2, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 3: batched_h2_ktile<OP, 3, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 4: batched_h2_ktile<OP, 4, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 5: batched_h2_ktile<OP, 5, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 6: batched_h2_ktile<OP, 6, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    case 7: batched_h2_ktile<OP, 7, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
    default: batched_h2_ktile<OP, 8, Q>(acc, As, Bs, ty, tx, cbase, swz, qn); break;
  }
}

// The persistent batched closure on the FP16 copies: the scheduling, TMA
// staging, padding skips, change test and proxy fence of
// closure_batched_kernel, with 64-k tiles of halves and k-pair words.
template <int OP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    closure_batched_h2_kernel(BatchGraph* graphs, const BatchMaps* __restrict__ maps, const int* order, int count,
                              int* queue, int max_iter, int conv_mode, const int* fp16_bad) {
  static_assert(OP == SIMD2_MAX_MIN || OP == SIMD2_MIN_MAX, "selection semirings only");
  constexpr int STAGES = kSimtStages;
  if (*fp16_bad != 0) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;
  __shared__ int s_graph;
  __shared__ int s_changed;
  __shared__ int s_failed;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int tx = lane & 15;
  const int ty = (warp & 7) * 2 + (lane >> 4);
  const int cbase = (warp >> 3) * 64;
  const int swz = ty & 7;
  const uint32_t ident = OP == SIMD2_MAX_MIN ? 0xfc00fc00u : 0x7c007c00u;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kSimtWarps);
    }
    fence_mbar_init();
    s_failed = 0;
  }
  __syncthreads();
  uint32_t gk = 0;  // running k-tile counter across tiles, steps and graphs

  while (true) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(queue, 1);
      s_graph = (q < count && !s_failed) ? order[q] : -1;
    }
    __syncthreads();
    const int gi = s_graph;
    if (gi < 0) break;
    BatchGraph& G = graphs[gi];
    const BatchMaps* mp = maps + gi;
    const int n = G.n, Kh = G.Kh, Np = G.Np;
    const int tiles_m = G.Mp / kBM, tiles_n = Np / kBN, ktiles = Kh / kH2BK;
    int it = 0, changed_any = 1;
    while (changed_any && it < max_iter) {
      const int cur = it & 1, nxt = cur ^ 1;
      const __half* X = G.Xh[cur];
      __half* Xn = G.Xh[nxt];
      __half* Pn = reinterpret_cast<__half*>(G.Ph[nxt]);
      const CUtensorMap* tmA = &mp->ah[cur];
      const CUtensorMap* tmB = &mp->bh[cur];
      if (threadIdx.x == 0) s_changed = 0;
      __syncthreads();
      int changed = 0;
      const int ntiles = tiles_m * tiles_n;
      const int nloads = ntiles * ktiles;
      auto issue = [&](int j) {
        const uint32_t g = gk + j;
        const int s = g % STAGES;
        if (!mbar_wait(&empty[s], ((g / STAGES) & 1) ^ 1)) {
          report_timeout(25);
          s_failed = 1;
        }
        const int tile = j / ktiles, kk = j - tile * ktiles;
        uint8_t* sa = smem + s * kStageBytes;
        mbar_arrive_expect_tx(&full[s], kStageBytes);
        tma_load_2d(sa, tmA, &full[s], kk * kH2BK, (tile % tiles_m) * kBM);
        tma_load_2d(sa + kATileBytes, tmB, &full[s], (tile / tiles_m) * kBN, kk * (kH2BK / 2));
      };
      if (threadIdx.x == 0)
        for (int j = 0; j < min(STAGES, nloads); j++) issue(j);
      for (int t = 0; t < ntiles; t++) {
        const int m0 = (t % tiles_m) * kBM;
        const int n0 = (t / tiles_m) * kBN;
        const int row_groups = min(8, (n - m0 + 15) / 16);
        const bool idle_cols = n0 + 64 >= n && cbase == 64;
        uint32_t acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = ident;
        for (int i = 0; i < ktiles; i++) {
          const int j = t * ktiles + i;
          const uint32_t g = gk + j;
          const int s = g % STAGES;
          if (threadIdx.x == 0 && j >= 1 && j - 1 + STAGES < nloads) issue(j - 1 + STAGES);
          if (!mbar_wait(&full[s], (g / STAGES) & 1)) {
            report_timeout(26);
            s_failed = 1;
          }
          const uint8_t* As = smem + s * kStageBytes;
          const uint32_t* Bs = reinterpret_cast<const uint32_t*>(As + kATileBytes);
          if (!idle_cols) {
            // chunks of 8 k of this k-tile that hold graph columns
            const int qn = min(8, (n - i * kH2BK + 7) >> 3);
            if (qn == 8) batched_h2_rows<OP, 8>(row_groups, acc, As, Bs, ty, tx, cbase, swz, qn);
            else batched_h2_rows<OP, 0>(row_groups, acc, As, Bs, ty, tx, cbase, swz, qn);
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[s]);
        }
        // epilogue: X_{t+1} = X_t (+) acc in both FP16 layouts (exact: every
        // value is an input entry or an identity), change test against X_t.
        // The 32 old values are loaded first, as 4-byte half pairs (col even,
        // Kh a multiple of 64), all in flight together.
        uint32_t oldw[8][2];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int row = m0 + ty + 16 * i;
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const int col0 = n0 + cbase + 32 * c + 2 * tx;
            oldw[i][c] = (row < n && col0 < n)
                             ? __ldcg(reinterpret_cast<const unsigned int*>(X + (long long)row * Kh + col0))
                             : 0u;
          }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int row = m0 + ty + 16 * i;
          if (row < n) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
              const int col0 = n0 + cbase + 32 * c + 2 * tx;
#pragma unroll
              for (int e = 0; e < 2; e++) {
                const int col = col0 + e;
                if (col < n) {
                  const uint32_t w = acc[i][2 * c + e];
                  const float lo = __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
                  const float hi = __half2float(__ushort_as_half((unsigned short)(w >> 16)));
                  const float old_v =
                      __half2float(__ushort_as_half((unsigned short)(e == 0 ? oldw[i][c] & 0xffffu : oldw[i][c] >> 16)));
                  const float v = Semiring<OP>::add(Semiring<OP>::add(lo, hi), old_v);
                  if (conv_changed(conv_mode, old_v, v)) changed = 1;
                  const __half vh = __float2half_rn(v);
                  Xn[(long long)row * Kh + col] = vh;
                  Pn[(long long)(row >> 1) * (2LL * Np) + 2 * col + (row & 1)] = vh;
                }
              }
            }
          }
        }
      }
      gk += nloads;
      if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(&s_changed, 1);
      // X_{t+1} was written through the generic proxy; the next step reads it with TMA.
      fence_proxy_async_global();
      __syncthreads();
      changed_any = s_changed && !s_failed;
      it++;
    }
    if (threadIdx.x == 0) {
      G.iters = it;
      G.changed = changed_any || s_failed;
    }
    __syncthreads();
  }
}

}  // namespace simd2
