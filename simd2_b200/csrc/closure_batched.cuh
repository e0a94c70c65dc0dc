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
  float* user;  // caller's matrix (result is copied back here)
  long long ldu;
  int iters;    // out: steps run (including the final unchanged one)
  int changed;  // out: 1 if the last step still changed something
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stage one k-tile (A rows m0..m0+127, k kt*32..+31; P rows kt*16..+15,
// floats 2*n0..2*n0+255) into shared memory with the same layout the TMA path
// produces: A with the 128-byte swizzle (16-byte chunk c of row r stored at
// chunk c ^ (r & 7)), P dense.
__device__ __forceinline__ void batch_stage_load(uint8_t* st, const float* X, int Kp, const float* P, int Np, int m0,
                                                 int n0, int kt) {
  float* As = reinterpret_cast<float*>(st);
  float* Bs = reinterpret_cast<float*>(st + kATileBytes);
  // A: 128 rows x 8 chunks of 16 bytes = 1024 copies
  for (int c = threadIdx.x; c < kBM * (kBK / 4); c += kSimtThreads) {
    const int r = c >> 3, q = c & 7;
    cp_async16(As + r * kBK + ((q ^ (r & 7)) << 2), X + (long long)(m0 + r) * Kp + kt * kBK + q * 4);
  }
  // P: 16 rows x 64 chunks = 1024 copies
  for (int c = threadIdx.x; c < (kBK / 2) * (2 * kBN / 4); c += kSimtThreads) {
    const int r = c >> 6, q = c & 63;
    cp_async16(Bs + r * (2 * kBN) + q * 4, P + (long long)(kt * (kBK / 2) + r) * (2LL * Np) + 2 * n0 + q * 4);
  }
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Tensor maps of one graph, in device memory: A role X[0], X[1] ([Mp][Kp],
// 128 x 32 boxes, 128-byte swizzle) and B role P[0], P[1] ([Kp/2][2Np],
// 16 x 256 boxes).  Encoded once on the host when the plan is made.
struct BatchMaps {
  CUtensorMap a[2];
  CUtensorMap b[2];
};

// One k-tile of the 8 x 4 register tile; ROWS < 8 skips rows ty + 16i for
// i >= ROWS (tile rows 16 ROWS..127), used when those rows lie past the graph.
template <int OP, int ROWS>
__device__ __forceinline__ void batched_mac_ktile(float (&acc)[8][4], const float* As, const float* Bs, int ty,
                                                  int tx, int cbase, int swz) {
  constexpr int WN = 2;
#pragma unroll 2
  for (int q = 0; q < kBK / 4; q++) {
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

template <int OP>
__global__ void __launch_bounds__(kSimtThreads, 1)
    closure_batched_kernel(BatchGraph* graphs, const BatchMaps* __restrict__ maps, const int* order, int count,
                           int* queue, int max_iter, int conv_mode) {
  constexpr int STAGES = kSimtStages;
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
            switch (row_groups) {
              case 1: batched_mac_ktile<OP, 1>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 2: batched_mac_ktile<OP, 2>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 3: batched_mac_ktile<OP, 3>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 4: batched_mac_ktile<OP, 4>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 5: batched_mac_ktile<OP, 5>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 6: batched_mac_ktile<OP, 6>(acc, As, Bs, ty, tx, cbase, swz); break;
              case 7: batched_mac_ktile<OP, 7>(acc, As, Bs, ty, tx, cbase, swz); break;
              default: batched_mac_ktile<OP, 8>(acc, As, Bs, ty, tx, cbase, swz); break;
            }
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[s]);
        }
        // epilogue: X_{t+1} = X_t (+) acc in both layouts, change test against X_t
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
                  const float old_v = __ldcg(X + (long long)row * Kp + col + e);
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
// One CTA row per (graph, padded row); grid-stride over graphs.
__global__ void batched_prep_kernel(BatchGraph* graphs, int count) {
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

// Copy every result X[iters & 1] back into the caller's matrix.
__global__ void batched_finish_kernel(BatchGraph* graphs, int count) {
  for (int g = blockIdx.y; g < count; g += gridDim.y) {
    BatchGraph& G = graphs[g];
    const float* R = G.X[G.iters & 1];
    const int n = G.n, Kp = G.Kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
         t += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(t / n), j = (int)(t - (long long)i * n);
      G.user[(long long)i * G.ldu + j] = R[(long long)i * Kp + j];
    }
  }
}

}  // namespace simd2
