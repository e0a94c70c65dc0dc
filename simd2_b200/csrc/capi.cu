// capi.cu -- C ABI entry points of libsimd2 (see include/simd2.h).
//
// Host side of the engine: argument checks, per-(device, stream) workspace,
// TMA descriptor encoding, kernel dispatch and the closure driver loop.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <atomic>
#include <type_traits>
#include <utility>
#include <vector>

#include "common.cuh"
#include "prep.cuh"
#include "srgemm_simt.cuh"
#include "tc_gemm.cuh"
#include "tc_gemm2.cuh"
#include "closure_batched.cuh"
#include "mlp.cuh"
#include "knn.cuh"
#include "knn_fused.cuh"
#include "pred.cuh"
#include "spgemm.cuh"
#include "mst.cuh"

namespace simd2 {
namespace {

#define SIMD2_CUDA_TRY(expr)                       \
  do {                                             \
    cudaError_t err__ = (expr);                    \
    if (err__ != cudaSuccess) return SIMD2_ERR_CUDA; \
  } while (0)

constexpr size_t kAlign = 1024;
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline int round_up(int x, int a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// device capability check (once per device)
// ---------------------------------------------------------------------------
int check_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SIMD2_ERR_NO_DEVICE;
  static std::mutex mu;
  static std::map<int, int> checked;
  std::lock_guard<std::mutex> lk(mu);
  auto it = checked.find(dev);
  if (it != checked.end()) return it->second;
  int major = 0, minor = 0;
  int rc = SIMD2_OK;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess || major != 10 ||
      minor != 0)
    rc = SIMD2_ERR_NO_DEVICE;
  checked[dev] = rc;
  return rc;
}

// ---------------------------------------------------------------------------
// launch accounting: a running count of every kernel this library launched,
// and optional CUDA-event timing of the main srgemm kernels (recorded on the
// stream each kernel is launched on).
// ---------------------------------------------------------------------------
std::atomic<long long> g_launches{0};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;
std::vector<int> g_prof_kind;        // kernel family of each timed launch
std::vector<long long> g_prof_opsv;  // algorithmic ops of each timed launch
size_t g_prof_used = 0;
long long g_prof_ops = 0;
double g_prof_ms[4] = {};
long long g_prof_n[4] = {}, g_prof_k_ops[4] = {};

inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Kernel families reported separately by simd2_profile_result.
enum ProfKind { kProfSimt = 0, kProfTensor = 1, kProfBatched = 2 };

// Returns the event pair to bracket a main-kernel launch, or nullptr.
std::pair<cudaEvent_t, cudaEvent_t>* prof_slot(long long ops, int kind = kProfSimt) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return nullptr;
  if (g_prof_used == g_prof_events.size()) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return nullptr;
    g_prof_events.push_back({a, b});
    g_prof_kind.push_back(0);
    g_prof_opsv.push_back(0);
  }
  g_prof_ops += ops;
  g_prof_kind[g_prof_used] = kind;
  g_prof_opsv[g_prof_used] = ops;
  return &g_prof_events[g_prof_used++];
}

// ---------------------------------------------------------------------------
// workspace: one growable device buffer per (device, stream)
// ---------------------------------------------------------------------------
std::mutex g_ws_mu;
// (device, stream, slot) -> growable buffer.  Slot 0 is the workspace of
// every entry point; slot 1 holds the dense matrix of the sparse closure's
// dense phase while that phase's own calls use slot 0.
std::map<std::tuple<int, cudaStream_t, int>, std::pair<void*, size_t>> g_ws;

int get_workspace_slot(cudaStream_t stream, int slot, size_t bytes, void** out) {
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mu);
  auto& e = g_ws[{dev, stream, slot}];
  if (e.second < bytes) {
    if (e.first) {
      cudaStreamSynchronize(stream);
      cudaFree(e.first);
      e = {nullptr, 0};
    }
    const size_t nb = align_up(std::max(bytes, (size_t)1 << 20), (size_t)2 << 20);
    void* p = nullptr;
    if (cudaMalloc(&p, nb) != cudaSuccess) {
      cudaGetLastError();
      return SIMD2_ERR_ALLOC;
    }
    e = {p, nb};
  }
  *out = e.first;
  return SIMD2_OK;
}

int get_workspace(cudaStream_t stream, size_t bytes, void** out) { return get_workspace_slot(stream, 0, bytes, out); }

// ---------------------------------------------------------------------------
// TMA descriptors
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Row-major float matrix [rows][cols] with row pitch `pitch` elements.
int make_map_f32(CUtensorMap* map, const void* base, long long rows, long long cols, long long pitch, int box_cols,
                 int box_rows, CUtensorMapSwizzle swz, bool nan_fill) {
  auto fn = encode_fn();
  if (!fn) return SIMD2_ERR_CUDA;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  nan_fill ? CU_TENSOR_MAP_FLOAT_OOB_FILL_NAN_REQUEST_ZERO_FMA : CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SIMD2_OK : SIMD2_ERR_CUDA;
}

// Row-major matrix [rows][cols] of `esize`-byte elements, pitch in elements.
int make_map_2d(CUtensorMap* map, CUtensorMapDataType dt, int esize, const void* base, long long rows,
                long long cols, long long pitch, int box_cols, int box_rows, CUtensorMapSwizzle swz) {
  auto fn = encode_fn();
  if (!fn) return SIMD2_ERR_CUDA;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(pitch * esize)};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SIMD2_OK : SIMD2_ERR_CUDA;
}

inline int grid_for(long long items, int threads = 256) {
  long long b = (items + threads - 1) / threads;
  return (int)std::max(1LL, std::min(b, 148LL * 16));
}

bool is_float_op(int op) { return op >= 0 && op <= 8 && op != SIMD2_OR_AND; }
bool is_sum_op(int op) { return op == SIMD2_PLUS_MUL || op == SIMD2_MINUS_SQUARE; }

float add_identity(int op) {
  switch (op) {
    case SIMD2_MIN_PLUS: case SIMD2_MIN_MUL: case SIMD2_MIN_MAX: return __builtin_inff();
    case SIMD2_MAX_PLUS: case SIMD2_MAX_MIN: case SIMD2_MAX_MUL: return -__builtin_inff();
    default: return 0.0f;
  }
}

// Padding value for out-of-range k: NaN products vanish under min/max.
float pad_value(int op) { return is_sum_op(op) ? 0.0f : __builtin_nanf(""); }

// ---------------------------------------------------------------------------
// srgemm plan: workspace layout for one call
// ---------------------------------------------------------------------------
struct Plan {
  int Kp, Np;
  size_t bp_off, bp_bytes;  // interleaved B'
  size_t ap_off, ap_bytes;  // packed A (0 when TMA reads A in place)
  int Kh;                   // FP16 selection path: K padded to 64 (0 = path off)
  size_t ah_off, bh_off, flag_off;
  size_t total;
};

// `half` reserves the FP16 selection path's operands (max_min / min_max).
Plan make_plan(int M, int N, int K, bool pack_a, bool half = false) {
  Plan p{};
  p.Kp = round_up(std::max(K, 1), kBK);
  p.Np = round_up(std::max(N, 1), kBN);
  p.bp_off = 0;
  p.bp_bytes = align_up((size_t)p.Kp * p.Np * 4, kAlign);
  p.ap_off = p.bp_bytes;
  p.ap_bytes = pack_a ? align_up((size_t)M * p.Kp * 4, kAlign) : 0;
  p.total = p.ap_off + p.ap_bytes;
  if (half) {
    p.Kh = round_up(std::max(K, 1), kH2BK);
    p.ah_off = p.total;
    p.bh_off = p.ah_off + align_up((size_t)M * p.Kh * 2, kAlign);
    p.flag_off = p.bh_off + align_up((size_t)(p.Kh / 2) * p.Np * 4, kAlign);
    p.total = p.flag_off + kAlign;
  }
  return p;
}

bool selection_op(int op) { return op == SIMD2_MAX_MIN || op == SIMD2_MIN_MAX; }

bool a_tma_ok(const void* A, long long lda) {
  return (reinterpret_cast<uintptr_t>(A) % 16 == 0) && ((lda * 4) % 16 == 0);
}

// Kernel configuration of the CUDA-core path: split-K factor over a
// thread-block cluster (1, 2, 4, 8) and block skipping with occupancy maps.
struct SimtConfig {
  int split = 1;
  bool skip = false;
  const uint8_t* occA = nullptr;
  const uint8_t* occB = nullptr;
  bool count_ops = true;  // false when an alternative kernel of the same call already counts them
};

// The (x)-annihilator whose products equal the (+)-identity: blocks made only
// of it (or NaN) contribute nothing and may be skipped.  Defined for the four
// semirings where the (+)-identity annihilates (x); others never skip.
bool skip_supported(int op) {
  return op == SIMD2_MIN_PLUS || op == SIMD2_MAX_PLUS || op == SIMD2_MAX_MIN || op == SIMD2_MIN_MAX;
}
float annihilator(int op) {
  return (op == SIMD2_MIN_PLUS || op == SIMD2_MIN_MAX) ? __builtin_inff() : -__builtin_inff();
}

template <int OP, int SPLIT, bool SKIP>
int launch_simt_cfg(int M, int N, int K, const CUtensorMap& mA, const CUtensorMap& mB, const EpilogueArgs& ep,
                    const SimtConfig& cfg, cudaStream_t stream) {
  constexpr int STAGES = kSimtStages;
  auto kern = srgemm_simt_kernel<OP, STAGES, SPLIT, SKIP>;
  const size_t smem = simt_smem_bytes(STAGES);
  static bool configured[64] = {};  // per instantiation and device
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return SIMD2_ERR_NO_DEVICE;
  if (!configured[dev]) {
    SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (SPLIT > 1) SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    configured[dev] = true;
  }
  const int tiles_m = (M + kBM - 1) / kBM;
  const int tiles_n = (N + kBN - 1) / kBN;
  auto* ev = prof_slot(cfg.count_ops ? 2LL * M * N * K : 0LL);
  if (ev) cudaEventRecord(ev->first, stream);
  if constexpr (SPLIT == 1) {
    kern<<<tiles_m * tiles_n, kSimtThreads, smem, stream>>>(mA, mB, M, N, K, ep, tiles_m, tiles_n, cfg.occA,
                                                            cfg.occB);
  } else {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(tiles_m * tiles_n * SPLIT);
    lc.blockDim = dim3(kSimtThreads);
    lc.dynamicSmemBytes = smem;
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = SPLIT;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    SIMD2_CUDA_TRY(cudaLaunchKernelEx(&lc, kern, mA, mB, M, N, K, ep, tiles_m, tiles_n, cfg.occA, cfg.occB));
  }
  count_launch();
  if (ev) cudaEventRecord(ev->second, stream);
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

template <int OP, bool SKIP>
int launch_simt_split(int M, int N, int K, const CUtensorMap& mA, const CUtensorMap& mB, const EpilogueArgs& ep,
                      const SimtConfig& cfg, cudaStream_t stream) {
  switch (cfg.split) {
    case 1: return launch_simt_cfg<OP, 1, SKIP>(M, N, K, mA, mB, ep, cfg, stream);
    case 2: return launch_simt_cfg<OP, 2, SKIP>(M, N, K, mA, mB, ep, cfg, stream);
    case 4: return launch_simt_cfg<OP, 4, SKIP>(M, N, K, mA, mB, ep, cfg, stream);
    case 8: return launch_simt_cfg<OP, 8, SKIP>(M, N, K, mA, mB, ep, cfg, stream);
    default: return SIMD2_ERR_INVALID_ARG;
  }
}

template <int OP>
int launch_simt(int M, int N, int K, const CUtensorMap& mA, const CUtensorMap& mB, const EpilogueArgs& ep,
                const SimtConfig& cfg, cudaStream_t stream) {
  if constexpr (OP == SIMD2_MIN_PLUS || OP == SIMD2_MAX_PLUS || OP == SIMD2_MAX_MIN || OP == SIMD2_MIN_MAX) {
    if (cfg.skip && cfg.occA && cfg.occB) return launch_simt_split<OP, true>(M, N, K, mA, mB, ep, cfg, stream);
  }
  return launch_simt_split<OP, false>(M, N, K, mA, mB, ep, cfg, stream);
}

int dispatch_simt(int op, int M, int N, int K, const CUtensorMap& mA, const CUtensorMap& mB, const EpilogueArgs& ep,
                  const SimtConfig& cfg, cudaStream_t stream) {
  switch (op) {
    case SIMD2_MIN_PLUS: return launch_simt<SIMD2_MIN_PLUS>(M, N, K, mA, mB, ep, cfg, stream);
    case SIMD2_MAX_PLUS: return launch_simt<SIMD2_MAX_PLUS>(M, N, K, mA, mB, ep, cfg, stream);
    case SIMD2_MAX_MIN: return launch_simt<SIMD2_MAX_MIN>(M, N, K, mA, mB, ep, cfg, stream);
    case SIMD2_MAX_MUL: return launch_simt<SIMD2_MAX_MUL>(M, N, K, mA, mB, ep, cfg, stream);
    case SIMD2_MIN_MUL: return launch_simt<SIMD2_MIN_MUL>(M, N, K, mA, mB, ep, cfg, stream);
    case SIMD2_MIN_MAX: return launch_simt<SIMD2_MIN_MAX>(M, N, K, mA, mB, ep, cfg, stream);
    default: return SIMD2_ERR_UNSUPPORTED;
  }
}

// ---------------------------------------------------------------------------
// block occupancy (for skip lists and the cost-model features)
// ---------------------------------------------------------------------------
struct OccPlan {
  int brA, bcA, brB, bcB;  // 32 x 32 block grid of A (M x K) and B (K x N)
  int tiles_m, tiles_n, ktiles;
  size_t occ32A, occ32B, occA, occB, stats, rowcnt, colcnt, total;
};

// Grid of occupancy_strip_kernel over a rows x cols matrix.
inline dim3 strip_grid(int rows, int cols) {
  return dim3((unsigned)((cols + kOccCols - 1) / kOccCols), (unsigned)((rows + kOccRows - 1) / kOccRows));
}

OccPlan make_occ_plan(int M, int N, int K, bool same) {
  OccPlan o{};
  o.brA = (M + 31) / 32;
  o.bcA = (K + 31) / 32;
  o.brB = (K + 31) / 32;
  o.bcB = (N + 31) / 32;
  o.tiles_m = (M + kBM - 1) / kBM;
  o.tiles_n = (N + kBN - 1) / kBN;
  o.ktiles = (K + kBK - 1) / kBK;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t r = off; off += align_up(std::max(bytes, (size_t)1), 256); return r; };
  o.occ32A = take((size_t)o.brA * o.bcA);
  o.occ32B = same ? o.occ32A : take((size_t)o.brB * o.bcB);
  o.occA = take((size_t)o.tiles_m * o.ktiles);
  o.occB = take((size_t)o.ktiles * o.tiles_n);
  o.stats = take(8 * sizeof(unsigned long long));
  o.rowcnt = take((size_t)std::max(M, K) * sizeof(int));
  o.colcnt = take((size_t)std::max(N, K) * sizeof(int));
  o.total = off;
  return o;
}

// Fills occA / occB and stats = {surviving (tm,tn,kt) triples, occupied A
// blocks, occupied B blocks}.  When `same`, A and B are the same matrix
// (closure), and one 32 x 32 pass serves both.
int compute_occupancy(int op, int M, int N, int K, const float* A, long long lda, const float* B, long long ldb,
                      bool same, uint8_t* base, const OccPlan& o, cudaStream_t stream) {
  const float ann = annihilator(op);
  auto* occ32A = base + o.occ32A;
  auto* occ32B = base + o.occ32B;
  occupancy_strip_kernel<false><<<strip_grid(M, K), 256, 0, stream>>>(A, lda, M, K, ann, ann, occ32A, o.bcA, nullptr,
                                                                      nullptr);
  count_launch();
  if (!same) {
    occupancy_strip_kernel<false><<<strip_grid(K, N), 256, 0, stream>>>(B, ldb, K, N, ann, ann, occ32B, o.bcB,
                                                                        nullptr, nullptr);
    count_launch();
  }
  auto* stats = reinterpret_cast<unsigned long long*>(base + o.stats);
  SIMD2_CUDA_TRY(cudaMemsetAsync(stats, 0, 8 * sizeof(unsigned long long), stream));
  occupancy_panels_kernel<<<std::min(o.ktiles, 148 * 4), 256, 0, stream>>>(
      occ32A, o.bcA, o.brA, occ32B, o.bcB, o.brB, o.tiles_m, o.tiles_n, o.ktiles, base + o.occA, base + o.occB, stats);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// The statistics of a closure step's X (n x n, A = B = X) that the cost
// model reads: the block occupancy (skip lists and stats[0..2]) and the
// stored entries / Gustavson products (stats[3], stats[4]), in one pass over X.
int compute_step_stats(int op, int n, const float* X, long long ldx, uint8_t* base, const OccPlan& o,
                       cudaStream_t stream) {
  auto* stats = reinterpret_cast<unsigned long long*>(base + o.stats);
  int* rowcnt = reinterpret_cast<int*>(base + o.rowcnt);
  int* colcnt = reinterpret_cast<int*>(base + o.colcnt);
  SIMD2_CUDA_TRY(cudaMemsetAsync(stats, 0, 8 * sizeof(unsigned long long), stream));
  SIMD2_CUDA_TRY(cudaMemsetAsync(rowcnt, 0, (size_t)n * sizeof(int), stream));
  SIMD2_CUDA_TRY(cudaMemsetAsync(colcnt, 0, (size_t)n * sizeof(int), stream));
  occupancy_strip_kernel<true><<<strip_grid(n, n), 256, 0, stream>>>(X, ldx, n, n, annihilator(op), add_identity(op),
                                                                     base + o.occ32A, o.bcA, rowcnt, colcnt);
  occupancy_panels_kernel<<<std::min(o.ktiles, 148 * 4), 256, 0, stream>>>(
      base + o.occ32A, o.bcA, o.brA, base + o.occ32A, o.bcA, o.brA, o.tiles_m, o.tiles_n, o.ktiles, base + o.occA,
      base + o.occB, stats);
  count_products_kernel<<<grid_for(n), 256, 0, stream>>>(n, rowcnt, colcnt, stats);
  for (int i = 0; i < 3; i++) count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// FP16 selection path (max_min / min_max): on the device, check that A and B
// hold only FP16 values; if so the packed-half kernel runs, else the FP32
// kernel (both are enqueued, each gated by one of the two flags, so the call
// stays asynchronous).  Same bits either way.
int enqueue_half_path(int op, int M, int N, int K, const float* A, long long lda, const float* B, long long ldb,
                      const EpilogueArgs& ep, uint8_t* ws, const Plan& plan, cudaStream_t stream) {
  int* flags = reinterpret_cast<int*>(ws + plan.flag_off);
  auto* Ah = reinterpret_cast<__half*>(ws + plan.ah_off);
  auto* Bh = reinterpret_cast<__half2*>(ws + plan.bh_off);
  // the FP16 copies are made unconditionally and clear flags[0] when an entry
  // is not exactly an FP16 value; then flags[1] = !flags[0] gates the FP32 path
  fp16_flags_init_kernel<<<1, 1, 0, stream>>>(flags);
  pack_half_rows_kernel<<<grid_for((long long)M * plan.Kh / 8), 256, 0, stream>>>(A, lda, M, K, Ah, plan.Kh, ep.gate,
                                                                              flags);
  interleave_half_kernel<<<grid_for((long long)(plan.Kh / 2) * plan.Np / 4), 256, 0, stream>>>(B, ldb, K, N, Bh, plan.Kh,
                                                                                            plan.Np, ep.gate, flags);
  fp16_flags_finish_kernel<<<1, 1, 0, stream>>>(flags);
  for (int i = 0; i < 4; i++) count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  CUtensorMap mA, mB;
  int rc = make_map_2d(&mA, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, Ah, M, plan.Kh, plan.Kh, kH2BK, kBM,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc) return rc;
  rc = make_map_2d(&mB, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, Bh, plan.Kh / 2, plan.Np, plan.Np, kBN, kH2BK / 2,
                   CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc) return rc;
  EpilogueArgs eh = ep;
  eh.gate2 = flags;
  const int tiles_m = (M + kBM - 1) / kBM;
  const int tiles_n = (N + kBN - 1) / kBN;
  const size_t smem = simt_smem_bytes(kSimtStages);
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  static bool configured[2][64] = {};
  const int which = op == SIMD2_MAX_MIN ? 0 : 1;
  auto kern = op == SIMD2_MAX_MIN ? srgemm_h2_kernel<SIMD2_MAX_MIN> : srgemm_h2_kernel<SIMD2_MIN_MAX>;
  if (dev < 0 || dev >= 64) return SIMD2_ERR_NO_DEVICE;
  if (!configured[which][dev]) {
    SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured[which][dev] = true;
  }
  auto* ev = prof_slot(2LL * M * N * K);
  if (ev) cudaEventRecord(ev->first, stream);
  kern<<<tiles_m * tiles_n, kSimtThreads, smem, stream>>>(mA, mB, M, N, K, eh, tiles_m, tiles_n);
  count_launch();
  if (ev) cudaEventRecord(ev->second, stream);
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// Core float srgemm with an explicit workspace.  T/MODE describe how A and B
// are read (float as-is, or any type normalised to {0,1}).
template <typename T, int MODE>
int srgemm_core(int op, int M, int N, int K, const T* A, long long lda, const T* B, long long ldb,
                const EpilogueArgs& ep, uint8_t* ws, const Plan& plan, bool pack_a, cudaStream_t stream,
                const SimtConfig& cfg = SimtConfig()) {
  const float pad = pad_value(op);
  float* Bp = reinterpret_cast<float*>(ws + plan.bp_off);
  const int* path_gate = nullptr;  // gates the FP32 path when the FP16 path is enqueued too
  if constexpr (MODE == 0 && std::is_same<T, float>::value) {
    if (plan.Kh > 0 && selection_op(op) && cfg.split == 1 && !cfg.skip) {
      int rc = enqueue_half_path(op, M, N, K, A, lda, B, ldb, ep, ws, plan, stream);
      if (rc) return rc;
      path_gate = reinterpret_cast<const int*>(ws + plan.flag_off) + 1;
    }
  }
  EpilogueArgs ep32 = ep;
  ep32.gate2 = path_gate;
  SimtConfig cfg32 = cfg;
  if (path_gate) cfg32.count_ops = false;  // the FP16 kernel's slot carries the operation count
  interleave_pairs_kernel<T, MODE><<<grid_for((long long)plan.Kp / 2 * plan.Np / 4), 256, 0, stream>>>(
      B, ldb, K, N, Bp, plan.Kp, plan.Np, pad, ep.gate, path_gate);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  const void* a_base = A;
  long long a_pitch = lda;
  if (pack_a) {
    float* Ap = reinterpret_cast<float*>(ws + plan.ap_off);
    pack_rows_kernel<T, MODE><<<grid_for((long long)M * plan.Kp), 256, 0, stream>>>(A, lda, M, K, Ap, plan.Kp, pad,
                                                                                    ep.gate, path_gate);
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    a_base = Ap;
    a_pitch = plan.Kp;
  }
  CUtensorMap mA, mB;
  int rc = make_map_f32(&mA, a_base, M, pack_a ? plan.Kp : K, a_pitch, kBK, kBM, CU_TENSOR_MAP_SWIZZLE_128B,
                        !is_sum_op(op));
  if (rc) return rc;
  rc = make_map_f32(&mB, Bp, plan.Kp / 2, 2LL * plan.Np, 2LL * plan.Np, 2 * kBN, kBK / 2, CU_TENSOR_MAP_SWIZZLE_NONE,
                    false);
  if (rc) return rc;
  return dispatch_simt(op, M, N, K, mA, mB, ep32, cfg32, stream);
}

// ---------------------------------------------------------------------------
// tensor-core paths
// ---------------------------------------------------------------------------
// TMA box width (elements along K) and swizzle of the tensor-core operand tiles.
template <int KIND>
constexpr int tc_box_k() { return TcCfg<KIND>::kBK; }
template <int KIND>
constexpr CUtensorMapSwizzle tc_swizzle() {
  return TcCfg<KIND>::kRowBytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
}

template <int KIND>
int launch_tc(int M, int N, int K, const CUtensorMap& a0, const CUtensorMap& a1, const CUtensorMap& b0,
              const CUtensorMap& b1, const TcEpilogue& ep, cudaStream_t stream) {
  auto kern = tc_gemm_kernel<KIND>;
  const size_t smem = tc_smem_bytes<KIND>();
  static bool configured[64] = {};
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return SIMD2_ERR_NO_DEVICE;
  if (!configured[dev]) {
    SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured[dev] = true;
  }
  const int tiles_m = (M + kTcBM - 1) / kTcBM;
  const int tiles_n = (N + kTcBN - 1) / kTcBN;
  auto* ev = prof_slot(2LL * M * N * K, kProfTensor);
  if (ev) cudaEventRecord(ev->first, stream);
  // persistent: at most one CTA per SM (shared memory and TMEM hold one)
  int sms = 148;
  SIMD2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = std::min(tiles_m * tiles_n, sms);
  kern<<<grid, kTcThreads, smem, stream>>>(a0, a1, b0, b1, M, N, K, ep, tiles_m, tiles_n);
  count_launch();
  if (ev) cudaEventRecord(ev->second, stream);
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// Pair tiles (256 x 256) from which the SM-pair kernel is used: enough to
// keep the pairs of the GPU busy; smaller problems run on single SMs.
constexpr int kTc2MinTiles = 64;

inline bool use_tc2(int M, int N) {
  return (long long)((M + kTc2BM - 1) / kTc2BM) * ((N + kTcBN - 1) / kTcBN) >= kTc2MinTiles;
}

// SM-pair launch: clusters of 2 CTAs, one pair per pair of SMs at most.
template <int KIND>
int launch_tc2(int M, int N, int K, const CUtensorMap& a0, const CUtensorMap& a1, const CUtensorMap& b0,
               const CUtensorMap& b1, const CUtensorMap& bh0, const CUtensorMap& bh1, const TcEpilogue& ep,
               cudaStream_t stream) {
  auto kern = tc_gemm2_kernel<KIND>;
  const size_t smem = tc2_smem_bytes<KIND>();
  static int max_pairs[64] = {};
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return SIMD2_ERR_NO_DEVICE;
  cudaLaunchConfig_t lc = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  lc.blockDim = dim3(kTcThreads);
  lc.dynamicSmemBytes = smem;
  lc.stream = stream;
  if (!max_pairs[dev]) {
    SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lc.gridDim = dim3(2 * 74);
    int clusters = 0;
    SIMD2_CUDA_TRY(cudaOccupancyMaxActiveClusters(&clusters, kern, &lc));
    max_pairs[dev] = std::max(1, clusters);
  }
  const int tiles_m = (M + kTc2BM - 1) / kTc2BM;
  const int tiles_n = (N + kTcBN - 1) / kTcBN;
  const int pairs = std::min(tiles_m * tiles_n, max_pairs[dev]);
  lc.gridDim = dim3(2 * pairs);
  auto* ev = prof_slot(2LL * M * N * K, kProfTensor);
  if (ev) cudaEventRecord(ev->first, stream);
  SIMD2_CUDA_TRY(cudaLaunchKernelEx(&lc, kern, a0, a1, b0, b1, bh0, bh1, M, N, K, ep, tiles_m, tiles_n));
  count_launch();
  if (ev) cudaEventRecord(ev->second, stream);
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

struct TcPlan {
  int Kp;
  size_t a0, a1, b0, b1, na, nb, nb64, total;
};

// bf16 hi/lo operands (plus_mul, minus_square)
TcPlan tc_plan_bf16(int M, int N, int K) {
  TcPlan p{};
  p.Kp = round_up(std::max(K, 1), 8);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  p.a0 = take((size_t)M * p.Kp * 2);
  p.a1 = take((size_t)M * p.Kp * 2);
  p.b0 = take((size_t)N * p.Kp * 2);
  p.b1 = take((size_t)N * p.Kp * 2);
  p.na = take((size_t)M * 4);
  p.nb = take((size_t)N * 4);
  p.nb64 = take((size_t)N * 8);
  p.total = off;
  return p;
}

// 0/1 byte operands (or_and)
TcPlan tc_plan_u8(int M, int N, int K) {
  TcPlan p{};
  p.Kp = round_up(std::max(K, 1), 16);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  p.a0 = take((size_t)M * p.Kp);
  p.b0 = take((size_t)N * p.Kp);
  p.a1 = p.a0;
  p.b1 = p.b0;
  p.na = p.nb = p.nb64 = 0;
  p.total = off;
  return p;
}

// Band of the minus_square exact recompute: distances below 2^-6 of |a|^2+|b|^2.
constexpr float kMinusSquareBand = 1.0f / 64.0f;

int srgemm_tc_sum(int op, int M, int N, int K, const float* A, long long lda, const float* B, long long ldb,
                  const float* C, long long ldc, float* D, long long ldd, int do_epilogue, uint8_t* ws,
                  const TcPlan& plan, cudaStream_t stream) {
  const int Kp = plan.Kp;
  auto* ahi = reinterpret_cast<__nv_bfloat16*>(ws + plan.a0);
  auto* alo = reinterpret_cast<__nv_bfloat16*>(ws + plan.a1);
  split_rows_bf16_kernel<<<grid_for((long long)M * Kp / 8), 256, 0, stream>>>(A, lda, M, K, ahi, alo, Kp);
  count_launch();
  float* na = reinterpret_cast<float*>(ws + plan.na);
  float* nb = reinterpret_cast<float*>(ws + plan.nb);
  double* nb64 = op == SIMD2_MINUS_SQUARE ? reinterpret_cast<double*>(ws + plan.nb64) : nullptr;
  if (nb64) SIMD2_CUDA_TRY(cudaMemsetAsync(nb64, 0, sizeof(double) * N, stream));
  dim3 tgrid((N + 31) / 32, (Kp + 31) / 32), tblock(32, 8);
  transpose_prep_kernel<float, 0><<<tgrid, tblock, 0, stream>>>(B, ldb, K, N, ws + plan.b0, ws + plan.b1, Kp, nb64);
  count_launch();
  if (op == SIMD2_MINUS_SQUARE) {
    row_norms_kernel<<<grid_for((long long)M * 32), 256, 0, stream>>>(A, lda, M, K, na);
    count_launch();
    round_norms_kernel<<<grid_for(N), 256, 0, stream>>>(nb64, N, nb);
    count_launch();
  }
  SIMD2_CUDA_TRY(cudaGetLastError());
  CUtensorMap ma0, ma1, mb0, mb1;
  const auto BF = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const auto SW = tc_swizzle<0>();
  constexpr int BX = tc_box_k<0>();
  int rc;
  // the SM-pair kernel stages B in halves of 128 rows
  const bool pair = use_tc2(M, N);
  const int brows = pair ? 128 : kTcBN;
  if ((rc = make_map_2d(&ma0, BF, 2, ahi, M, Kp, Kp, BX, kTcBM, SW))) return rc;
  if ((rc = make_map_2d(&ma1, BF, 2, alo, M, Kp, Kp, BX, kTcBM, SW))) return rc;
  if ((rc = make_map_2d(&mb0, BF, 2, ws + plan.b0, N, Kp, Kp, BX, brows, SW))) return rc;
  if ((rc = make_map_2d(&mb1, BF, 2, ws + plan.b1, N, Kp, Kp, BX, brows, SW))) return rc;
  // the pair kernel's half tiles stage 64 rows of B^T per CTA
  CUtensorMap mbh0 = mb0, mbh1 = mb1;
  if (pair) {
    if ((rc = make_map_2d(&mbh0, BF, 2, ws + plan.b0, N, Kp, Kp, BX, 64, SW))) return rc;
    if ((rc = make_map_2d(&mbh1, BF, 2, ws + plan.b1, N, Kp, Kp, BX, 64, SW))) return rc;
  }
  TcEpilogue ep{};
  ep.op = op;
  ep.do_epilogue = do_epilogue;
  ep.C = do_epilogue ? (const void*)C : (const void*)D;
  ep.ldc = do_epilogue ? ldc : ldd;
  ep.D = D;
  ep.ldd = ldd;
  ep.norm_a = na;
  ep.norm_b = nb;
  ep.A32 = A;
  ep.lda32 = lda;
  ep.B32 = B;
  ep.ldb32 = ldb;
  ep.K = K;
  ep.band = kMinusSquareBand;
  if (pair) return launch_tc2<0>(M, N, K, ma0, ma1, mb0, mb1, mbh0, mbh1, ep, stream);
  return launch_tc<0>(M, N, K, ma0, ma1, mb0, mb1, ep, stream);
}

// delta (or_and closure, pair kernel only): the maps of TcEpilogue.
struct TcDelta {
  uint8_t* chg_row = nullptr;
  uint8_t* chg_col = nullptr;
  const uint8_t* need_row = nullptr;
  const uint8_t* need_col = nullptr;
};

template <typename T>
int srgemm_tc_orand(int M, int N, int K, const T* A, long long lda, const T* B, long long ldb, const T* C,
                    long long ldc, T* D, long long ldd, int do_epilogue, int* changed, uint8_t* ws,
                    const TcPlan& plan, cudaStream_t stream, const TcDelta& delta = TcDelta()) {
  const int Kp = plan.Kp;
  uint8_t* a8 = ws + plan.a0;
  uint8_t* b8 = ws + plan.b0;
  bool_rows_u8_kernel<T><<<grid_for((long long)M * Kp / 16), 256, 0, stream>>>(A, lda, M, K, a8, Kp);
  count_launch();
  if constexpr (std::is_same_v<T, uint8_t>) {
    transpose_bool_u8_kernel<<<dim3((N + 63) / 64, (Kp + 63) / 64), 256, 0, stream>>>(B, ldb, K, N, b8, Kp);
  } else {
    dim3 tgrid((N + 31) / 32, (Kp + 31) / 32), tblock(32, 8);
    transpose_prep_kernel<T, 1><<<tgrid, tblock, 0, stream>>>(B, ldb, K, N, b8, nullptr, Kp);
  }
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  CUtensorMap ma, mb;
  const auto U8 = CU_TENSOR_MAP_DATA_TYPE_UINT8;
  const auto SW = CU_TENSOR_MAP_SWIZZLE_128B;
  int rc;
  const bool pair = use_tc2(M, N);
  if ((rc = make_map_2d(&ma, U8, 1, a8, M, Kp, Kp, 128, kTcBM, SW))) return rc;
  if ((rc = make_map_2d(&mb, U8, 1, b8, N, Kp, Kp, 128, pair ? 128 : kTcBN, SW))) return rc;
  CUtensorMap mbh = mb;  // the pair kernel's half tiles stage 64 rows of B^T per CTA
  if (pair && (rc = make_map_2d(&mbh, U8, 1, b8, N, Kp, Kp, 128, 64, SW))) return rc;
  TcEpilogue ep{};
  ep.op = SIMD2_OR_AND;
  ep.do_epilogue = do_epilogue;
  ep.C = do_epilogue ? (const void*)C : (const void*)D;
  ep.ldc = do_epilogue ? ldc : ldd;
  ep.D = D;
  ep.ldd = ldd;
  ep.out_u8 = sizeof(T) == 1;
  ep.changed = changed;
  if (pair) {
    ep.chg_row = delta.chg_row;
    ep.chg_col = delta.chg_col;
    ep.need_row = delta.need_row;
    ep.need_col = delta.need_col;
    return launch_tc2<1>(M, N, K, ma, ma, mb, mb, mbh, mbh, ep, stream);
  }
  return launch_tc<1>(M, N, K, ma, ma, mb, mb, ep, stream);
}

int check_dims(int M, int N, int K, long long lda, long long ldb, long long ldc, long long ldd, const void* A,
               const void* B, const void* C, const void* D, int do_epilogue) {
  if (M < 0 || N < 0 || K < 0) return SIMD2_ERR_INVALID_ARG;
  if (M == 0 || N == 0) return SIMD2_OK;
  if (!D || ldd < N) return SIMD2_ERR_INVALID_ARG;
  if (K > 0 && (!A || !B || lda < K || ldb < N)) return SIMD2_ERR_INVALID_ARG;
  if (do_epilogue && (!C || ldc < N)) return SIMD2_ERR_INVALID_ARG;
  return SIMD2_OK;
}

// D = id (+) C for K == 0 (a copy of C for every semiring, id otherwise).
int srgemm_k0(int op, int M, int N, const float* C, long long ldc, float* D, long long ldd, int do_epilogue,
              cudaStream_t stream) {
  if (do_epilogue) {
    SIMD2_CUDA_TRY(cudaMemcpy2DAsync(D, ldd * 4, C, ldc * 4, (size_t)N * 4, M, cudaMemcpyDeviceToDevice, stream));
  } else {
    fill_kernel<float><<<grid_for((long long)M * N), 256, 0, stream>>>(D, ldd, M, N, add_identity(op));
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
  }
  return SIMD2_OK;
}

EpilogueArgs make_epilogue(const float* C, long long ldc, float* D, long long ldd, int do_epilogue, int* changed,
                           int conv) {
  EpilogueArgs ep{};
  ep.C = do_epilogue ? C : D;
  ep.ldc = do_epilogue ? ldc : ldd;
  ep.D = D;
  ep.ldd = ldd;
  ep.do_epilogue = do_epilogue;
  ep.vec2 = (reinterpret_cast<uintptr_t>(D) % 8 == 0) && (ldd % 2 == 0) &&
            (!do_epilogue || ((reinterpret_cast<uintptr_t>(C) % 8 == 0) && (ldc % 2 == 0)));
  ep.changed = changed;
  ep.conv_mode = conv;
  return ep;
}

int srgemm_f32_ws(int op, int M, int N, int K, const float* A, long long lda, const float* B, long long ldb,
                  const float* C, long long ldc, float* D, long long ldd, int do_epilogue, int* changed, int conv,
                  uint8_t* ws_or_null, cudaStream_t stream) {
  if (K == 0) return srgemm_k0(op, M, N, C, ldc, D, ldd, do_epilogue, stream);
  if (is_sum_op(op)) {
    const TcPlan tp = tc_plan_bf16(M, N, K);
    uint8_t* ws = ws_or_null;
    if (!ws) {
      void* p = nullptr;
      int rc = get_workspace(stream, tp.total, &p);
      if (rc) return rc;
      ws = static_cast<uint8_t*>(p);
    }
    return srgemm_tc_sum(op, M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, ws, tp, stream);
  }
  const bool pack_a = !a_tma_ok(A, lda);
  // the FP16 selection path needs workspace beyond the base plan, so it is
  // only planned when the library provides the workspace itself
  const Plan plan = make_plan(M, N, K, pack_a, ws_or_null == nullptr && selection_op(op));
  uint8_t* ws = ws_or_null;
  if (!ws) {
    void* p = nullptr;
    int rc = get_workspace(stream, plan.total, &p);
    if (rc) return rc;
    ws = static_cast<uint8_t*>(p);
  }
  const EpilogueArgs ep = make_epilogue(C, ldc, D, ldd, do_epilogue, changed, conv);
  return srgemm_core<float, 0>(op, M, N, K, A, lda, B, ldb, ep, ws, plan, pack_a, stream);
}

// or_and on the INT8 tensor cores (0/1 bytes, S32 counts), exact.
template <typename T>
int srgemm_orand(int M, int N, int K, const T* A, long long lda, const T* B, long long ldb, const T* C, long long ldc,
                 T* D, long long ldd, int do_epilogue, cudaStream_t stream) {
  int rc = check_dims(M, N, K, lda, ldb, ldc, ldd, A, B, C, D, do_epilogue);
  if (rc || M == 0 || N == 0) return rc;
  if ((rc = check_device())) return rc;
  if (K == 0) {
    // D = 0 (+) C
    if (do_epilogue) {
      bool_copy_kernel<T><<<grid_for((long long)M * N), 256, 0, stream>>>(C, ldc, D, ldd, M, N);
      count_launch();
    } else {
      fill_kernel<T><<<grid_for((long long)M * N), 256, 0, stream>>>(D, ldd, M, N, T(0));
      count_launch();
    }
    SIMD2_CUDA_TRY(cudaGetLastError());
    return SIMD2_OK;
  }
  const TcPlan plan = tc_plan_u8(M, N, K);
  void* p = nullptr;
  if ((rc = get_workspace(stream, plan.total, &p))) return rc;
  return srgemm_tc_orand<T>(M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, nullptr,
                            static_cast<uint8_t*>(p), plan, stream);
}

}  // namespace

// ---------------------------------------------------------------------------
// closure driver
// ---------------------------------------------------------------------------
namespace {

// Split-K factors the autotuner measured best for the dense closure step, by
// size: entry i applies from n = g_dense_n[i] up to the next entry's n (set by
// simd2_set_dense_configs; empty until then).
std::mutex g_dense_mu;
std::vector<int> g_dense_n, g_dense_split;

// Split-K factor of the dense path: the autotuned table's entry for n when
// one applies, else the largest power of two (at most 4) with
// tiles * split <= SM count, so small problems still fill the GPU.
int dense_split(int n, int sms) {
  {
    std::lock_guard<std::mutex> lk(g_dense_mu);
    int pick = 0;
    for (size_t i = 0; i < g_dense_n.size(); i++)
      if (g_dense_n[i] <= n) pick = g_dense_split[i];
    if (pick) return pick;
  }
  const long long tiles = (long long)((n + kBM - 1) / kBM) * ((n + kBN - 1) / kBN);
  int s = 1;
  while (s < 4 && tiles * s * 2 <= sms) s *= 2;
  return s;
}

constexpr int kOrAndSparseMinN = 8192;

// How a closure's sparse opening decides, step by step, whether the next
// squaring runs as a CSR SpGEMM step.  Every policy gives the same bits.
struct OpeningPolicy {
  // a step forming more products than this is never run sparse
  unsigned long long max_products = 0;
  // learned: the MLP in `mlp` compares the sparse step with the dense
  // configurations from the step's statistics (computed into the occupancy
  // workspace `obase` / `occ`); null: every step under max_products runs sparse
  const float* mlp = nullptr;
  uint8_t* obase = nullptr;
  const OccPlan* occ = nullptr;
  int* decision = nullptr;  // device int[1 + kSparseConfig + 1]
  int sms = 148;
  int can_skip = 0;
  float* step_feat = nullptr;  // optional: features of each opening step (kMlpFeat each)
};

// Defined with the SpGEMM host code below.
int closure_sparse_opening(int op, int n, float* X, long long ldx, int max_iter, const OpeningPolicy& pol,
                           int* steps, bool* changed, int* step_cfg, float* step_ms, cudaStream_t stream);
int closure_sparse_opening_u8(int n, uint8_t* X, long long ldx, int max_iter, int* steps, bool* changed,
                              cudaStream_t stream);

// Closure steps enqueued in chunks without a host round trip per step.
// changed[t] is written by step t; every kernel of step t+1 reads changed[t]
// as its gate and does nothing when it is 0, so steps enqueued past the fixed
// point cost only their launches.  The host reads the chunk's flags once.
int closure_gated(int op, int n, float* X, long long ldx, int max_iter, int conv, int fixed_cfg, bool fixed,
                  bool can_skip, bool need_occ, const OccPlan& occ, uint8_t* ws, size_t x_off, int* changed,
                  uint8_t* obase, int* iters_out, int* step_cfg, float* step_ms, int sms, cudaStream_t stream,
                  const float* A0 = nullptr, long long lda0 = 0) {
  int rc = SIMD2_OK;
  const int auto_split = dense_split(n, sms);
  float* bufs[2] = {X, reinterpret_cast<float*>(ws + x_off)};
  const long long lds[2] = {ldx, n};
  SIMD2_CUDA_TRY(cudaMemsetAsync(changed, 0, (size_t)(max_iter + 1) * sizeof(int), stream));
  std::vector<cudaEvent_t> evs;
  int done_at = -1;  // step index whose flag was 0 (converged), -1 while running
  int enq = 0;
  int chunk = 4;
  std::vector<int> h(max_iter);
  while (done_at < 0 && enq < max_iter && rc == SIMD2_OK) {
    const int first = enq;
    const int last = std::min(max_iter, enq + chunk);
    for (int t = first; t < last; t++) {
      float* cur = bufs[t & 1];
      float* nxt = bufs[(t + 1) & 1];
      const long long ldcur = lds[t & 1], ldnxt = lds[(t + 1) & 1];
      const int* gate = t > 0 ? changed + (t - 1) : nullptr;
      if (step_ms) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        evs.push_back(a);
        evs.push_back(b);
        cudaEventRecord(a, stream);
      }
      SimtConfig cfg;
      cfg.split = fixed ? config_split(fixed_cfg) : auto_split;
      cfg.skip = fixed && config_skip(fixed_cfg) && can_skip && need_occ;
      if (cfg.skip) {
        // occupancy of a gated-off step is harmless work on an unchanged matrix
        if ((rc = compute_occupancy(op, n, n, n, cur, ldcur, cur, ldcur, true, obase, occ, stream))) break;
        cfg.occA = obase + occ.occA;
        cfg.occB = obase + occ.occB;
      }
      if (step_cfg) step_cfg[t] = (cfg.skip ? 4 : 0) | (cfg.split == 1 ? 0 : cfg.split == 2 ? 1 : cfg.split == 4 ? 2 : 3);
      // A operand: X_t (repeated squaring) or the fixed adjacency A0 (Bellman-Ford form)
      const float* Aop = A0 ? A0 : cur;
      const long long lda_op = A0 ? lda0 : ldcur;
      const bool pk = !a_tma_ok(Aop, lda_op);
      const Plan pl = make_plan(n, n, n, pk, selection_op(op));
      EpilogueArgs ep = make_epilogue(cur, ldcur, nxt, ldnxt, 1, changed + t, conv);
      ep.gate = gate;
      if ((rc = srgemm_core<float, 0>(op, n, n, n, Aop, lda_op, cur, ldcur, ep, ws, pl, pk, stream, cfg))) break;
      if (step_ms) cudaEventRecord(evs.back(), stream);
    }
    if (rc) break;
    enq = last;
    if (cudaMemcpyAsync(h.data() + first, changed + first, sizeof(int) * (last - first), cudaMemcpyDeviceToHost,
                        stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
      rc = SIMD2_ERR_CUDA;
      break;
    }
    for (int t = first; t < last; t++)
      if (h[t] == 0) {
        done_at = t;
        break;
      }
    chunk = std::min(chunk * 2, 64);
  }
  const int iters = done_at >= 0 ? done_at + 1 : enq;
  if (rc == SIMD2_OK) {
    // result of the last executed step t = iters - 1 is in bufs[iters & 1]
    float* res = bufs[iters & 1];
    if (res != X)
      rc = cudaMemcpy2DAsync(X, ldx * 4, res, lds[iters & 1] * 4, (size_t)n * 4, n, cudaMemcpyDeviceToDevice,
                             stream) == cudaSuccess
               ? SIMD2_OK
               : SIMD2_ERR_CUDA;
  }
  if (cudaStreamSynchronize(stream) != cudaSuccess && rc == SIMD2_OK) rc = SIMD2_ERR_CUDA;
  if (step_ms) {
    for (int t = 0; t < iters && 2 * t + 1 < (int)evs.size(); t++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, evs[2 * t], evs[2 * t + 1]);
      step_ms[t] = ms;
    }
    for (auto e : evs) cudaEventDestroy(e);
  }
  if (rc) return rc;
  if (iters_out) *iters_out = iters;
  return done_at >= 0 ? SIMD2_OK : SIMD2_ERR_NOT_CONVERGED;
}

// Closure by repeated squaring with a per-step kernel configuration:
//   dispatch 0 (dense)  : no skip, split-K from the tile count (the plain path);
//   dispatch 1 (fixed)  : `fixed_cfg` every step: a dense configuration
//                         (split = 1 << (cfg & 3), skip = cfg >> 2), or
//                         kSparseConfig: CSR SpGEMM steps for as long as X fits
//                         the sparse store (under n^3/16 products), then the
//                         plain dense steps (used to record sparse-step times);
//   dispatch 2 (learned): per step, the statistics of X_t -> features -> the
//                         MLP `mlp_params` predicts the time of every dense
//                         configuration and, while X_t is sparse, of a CSR
//                         SpGEMM step; the cheapest one runs;
//   dispatch 3 (rules)  : the hand-written policy without the MLP: sparse
//                         steps while X_t holds at most n^2/32 entries and the
//                         step forms at most n^3/256 products, then `fixed_cfg`
//                         for every dense step.
// Every configuration computes the same bits, so the dispatch only moves time.
// step_cfg / step_ms / step_feat (host arrays of max_iter, max_iter,
// max_iter * kMlpFeat entries, each optional) record what each step ran, its
// device time (operand prep + srgemm, plus the occupancy pass of a skipping
// step; a sparse step's count and fill passes, the first one with X's
// conversion to CSR) and its features.
int closure_f32_ex(int op, int n, float* X, long long ldx, int max_iter, int conv, int dispatch, int fixed_cfg,
                   const float* mlp_params, int* iters_out, int* step_cfg, float* step_ms, float* step_feat,
                   cudaStream_t stream) {
  if (iters_out) *iters_out = 0;
  if (n < 0 || max_iter < 0 || !is_float_op(op) || is_sum_op(op) || (n > 0 && (!X || ldx < n)))
    return SIMD2_ERR_INVALID_ARG;
  if (dispatch < 0 || dispatch > 3 || (dispatch == 2 && !mlp_params) || fixed_cfg < 0 ||
      fixed_cfg > (dispatch == 1 ? kSparseConfig : kNumConfigs - 1))
    return SIMD2_ERR_INVALID_ARG;
  if (n == 0 || max_iter == 0) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  int sms = 148;
  {
    int dev = 0;
    SIMD2_CUDA_TRY(cudaGetDevice(&dev));
    SIMD2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  const bool fixed_sparse = dispatch == 1 && fixed_cfg == kSparseConfig;
  // A learned step costs a statistics pass, the MLP launch and a host round
  // trip (about 25 us together on B200).  Up to n = kLearnedMinN a whole dense
  // step costs about as much (2n^3 <= 2.1 Gop, under 70 us on 148 SMs), so no
  // choice can win back its decision and the plain gated path runs instead;
  // the rules policy does the same.
  if ((dispatch == 2 || dispatch == 3) && n <= kLearnedMinN) {
    dispatch = 0;
    if (step_feat) std::fill(step_feat, step_feat + (size_t)max_iter * kMlpFeat, 0.f);
    step_feat = nullptr;
  }
  const bool can_skip = skip_supported(op) && (n + kBK - 1) / kBK <= kMaxSkipKtiles;
  const bool opening = (dispatch == 2 || dispatch == 3 || fixed_sparse) && conv == SIMD2_CONV_EXACT;
  const bool fixed_skip = (dispatch == 1 || dispatch == 3) && fixed_cfg < kNumConfigs && config_skip(fixed_cfg);
  const bool need_occ = dispatch == 2 || step_feat != nullptr || (fixed_skip && can_skip);
  // Workspace: [srgemm plan][Xnew n x n][flag + decision][occupancy]
  const bool pack_a = !a_tma_ok(X, ldx) || (n % 4 != 0);
  const Plan plan = make_plan(n, n, n, pack_a, selection_op(op));
  const OccPlan occ = make_occ_plan(n, n, n, true);
  const size_t x_off = align_up(plan.total, kAlign);
  const size_t f_off = x_off + align_up((size_t)n * n * 4, kAlign);
  // flag word + learned decision (256 bytes), then one change flag per step
  const size_t o_off = f_off + align_up(256 + (size_t)(max_iter + 1) * sizeof(int), kAlign);
  // Delta steps (see srgemm_simt_kernel, SKIP): the learned and rules loops of
  // a min_plus / max_plus closure with the exact change test keep, per step,
  // which 32 x 32 blocks changed, in two ping-pong pairs of maps laid out as
  // the occupancy maps.  Recording runs (autotuner timings per configuration)
  // and fixed configurations keep the plain steps.
  const bool use_delta = (op == SIMD2_MIN_PLUS || op == SIMD2_MAX_PLUS) && conv == SIMD2_CONV_EXACT && can_skip &&
                         (dispatch == 2 || dispatch == 3) && step_feat == nullptr;
  const size_t cmA = align_up((size_t)occ.tiles_m * occ.ktiles, kAlign);
  const size_t cmB = align_up((size_t)occ.ktiles * occ.tiles_n, kAlign);
  const size_t c_off = o_off + (need_occ ? align_up(occ.total, kAlign) : 0);
  const size_t total = c_off + (use_delta ? 2 * (cmA + cmB) : 0);
  void* p = nullptr;
  if ((rc = get_workspace(stream, total, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  float* Xn = reinterpret_cast<float*>(ws + x_off);
  int* flag = reinterpret_cast<int*>(ws + f_off);
  int* decision = flag + 8;  // [0] config, [1 + c] prediction of config c
  uint8_t* obase = ws + o_off;
  uint8_t* chg[2][2] = {};  // [parity][A map, B map]
  if (use_delta)
    for (int q = 0; q < 2; q++) {
      chg[q][0] = ws + c_off + q * (cmA + cmB);
      chg[q][1] = chg[q][0] + cmA;
    }

  // The opening: sparse steps while X is sparse, under the dispatch's policy
  // (bitwise change test only).
  int it0 = 0;
  if (opening) {
    const unsigned long long n3 = (unsigned long long)n * (unsigned long long)n * (unsigned long long)n;
    OpeningPolicy pol;
    // A sparse step past n^3/16 products would cost at least 9x a dense step
    // at the measured rates (about 120 G products/s against 17 T MAC/s), so
    // neither the learned nor the recording policy considers it; the rules
    // policy keeps a step sparse only under n^3/256 (two thirds of a dense step).
    pol.max_products = dispatch == 3 ? n3 / 256ull : n3 / 16ull;
    if (dispatch == 2) {
      pol.mlp = mlp_params;
      pol.obase = obase;
      pol.occ = &occ;
      pol.decision = decision;
      pol.sms = sms;
      pol.can_skip = can_skip ? 1 : 0;
      pol.step_feat = step_feat;
    }
    bool ch = true;
    if (step_feat) std::fill(step_feat, step_feat + (size_t)max_iter * kMlpFeat, 0.f);
    if ((rc = closure_sparse_opening(op, n, X, ldx, max_iter, pol, &it0, &ch, step_cfg, step_ms, stream))) return rc;
    if (!ch || it0 == max_iter) {
      if (iters_out) *iters_out = it0;
      return ch ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
    }
    max_iter -= it0;
    if (step_cfg) step_cfg += it0;
    if (step_ms) step_ms += it0;
    if (step_feat) step_feat += (size_t)it0 * kMlpFeat;
    // Up to n = kLearnedLoopMinN a per-step choice (measured on R-MAT graphs)
    // gains less than its decisions cost: the gated dense path goes on.
    if ((dispatch == 2 || dispatch == 3) && n <= kLearnedLoopMinN) {
      dispatch = 0;
      if (step_feat) std::fill(step_feat, step_feat + (size_t)max_iter * kMlpFeat, 0.f);
      step_feat = nullptr;
    }
  }
  if (fixed_sparse) dispatch = 0;  // the dense steps after a recorded opening run the plain path

  const bool per_step = dispatch == 2 || dispatch == 3 || step_feat != nullptr;
  if (!per_step) {
    int it2 = 0;
    rc = closure_gated(op, n, X, ldx, max_iter, conv, fixed_cfg, dispatch == 1, can_skip, need_occ, occ, ws, x_off,
                       reinterpret_cast<int*>(ws + f_off + 256), obase, &it2, step_cfg, step_ms, sms, stream);
    if (iters_out) *iters_out = it0 + it2;
    return rc;
  }
  // Per-step loop (learned or rules dispatch, or feature recording): the
  // statistics and the cost-model choice for step t+1 are enqueued right after
  // step t's srgemm, so one host synchronisation per step reads step t's
  // change flag together with step t+1's decision (and features).
  const bool want_feat = dispatch == 2 || step_feat != nullptr;
  cudaEvent_t ev[4] = {};  // srgemm start/end, occupancy start/end
  if (step_ms)
    for (auto& e : ev) SIMD2_CUDA_TRY(cudaEventCreate(&e));
  float occ_ms = 0.f;
  auto enqueue_occ = [&](const float* m, long long ld) -> int {
    if (step_ms) cudaEventRecord(ev[2], stream);
    int r = want_feat ? compute_step_stats(op, n, m, ld, obase, occ, stream)
                      : compute_occupancy(op, n, n, n, m, ld, m, ld, true, obase, occ, stream);
    if (r) return r;
    if (dispatch == 2) {
      mlp_choose_kernel<<<1, 32, 0, stream>>>(mlp_params, reinterpret_cast<unsigned long long*>(obase + occ.stats), n,
                                              occ.tiles_m, occ.tiles_n, occ.ktiles, sms, can_skip ? 1 : 0, 8, 0,
                                              decision);
      count_launch();
    }
    if (step_ms) cudaEventRecord(ev[3], stream);
    return SIMD2_OK;
  };
  // host copies of {flag, decision[0..8]} and the step statistics
  int hbuf[9] = {};
  unsigned long long hst[5] = {};
  auto read_back = [&](bool want_flag, bool want_dec) -> int {
    if (want_flag || want_dec) {
      if (cudaMemcpyAsync(hbuf, flag, sizeof(hbuf), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return SIMD2_ERR_CUDA;
    }
    if (want_dec) {
      if (cudaMemcpyAsync(hst, obase + occ.stats, sizeof(hst), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return SIMD2_ERR_CUDA;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) return SIMD2_ERR_CUDA;
    if (step_ms && want_dec) cudaEventElapsedTime(&occ_ms, ev[2], ev[3]);
    return SIMD2_OK;
  };
  const int ds = dense_split(n, sms);
  const int default_cfg = dispatch == 1 || dispatch == 3 ? fixed_cfg : (ds == 1 ? 0 : ds == 2 ? 1 : 2);
  float* cur = X;
  long long ldcur = ldx;
  float* nxt = Xn;
  long long ldnxt = n;
  int it = 0;
  int changed = 1;
  int cfg_id = default_cfg;
  // Closure steps only fill X in: once every (tile, k-tile) block triple is
  // occupied, no later step can skip anything, so the learned and rules loops
  // stop the statistics pass and keep the split factor of the last choice
  // without skipping (feature recording keeps the pass).
  const unsigned long long all_triples = (unsigned long long)occ.tiles_m * occ.tiles_n * occ.ktiles;
  bool occ_on = need_occ;
  // occ_fresh: the occupancy maps hold this step's input; occ_full: every
  // block triple was occupied, so the maps are all ones and stay valid (a
  // closure only fills X in).  A delta step needs one or the other.
  bool occ_fresh = false, occ_full = false;
  bool prev_chg = false;  // the previous step wrote change maps (chg[par ^ 1])
  int par = 0;
  auto settle = [&]() {
    if ((dispatch == 2 || dispatch == 3) && !step_feat && hst[0] >= all_triples) {
      occ_on = false;
      occ_full = true;
      cfg_id &= 3;
    }
  };
  if (need_occ) {
    if ((rc = enqueue_occ(cur, ldcur)) || (rc = read_back(false, true))) return rc;
    occ_fresh = true;
    if (dispatch == 2) cfg_id = hbuf[8];  // decision[0]
    if (step_feat) mlp_features(n, occ.tiles_m, occ.tiles_n, occ.ktiles, hst, sms, step_feat);
    settle();
  }
  while (changed && it < max_iter) {
    SimtConfig cfg;
    cfg.split = config_split(cfg_id);
    const bool delta = use_delta && prev_chg && (occ_fresh || occ_full);
    cfg.skip = can_skip && ((config_skip(cfg_id) && occ_on) || delta);
    if (cfg.skip) {
      cfg.occA = obase + occ.occA;
      cfg.occB = obase + occ.occB;
    }
    if (step_cfg) step_cfg[it] = (cfg.skip ? 4 : 0) | (cfg.split == 1 ? 0 : cfg.split == 2 ? 1 : cfg.split == 4 ? 2 : 3);
    const float step_occ_ms = (occ_on && cfg.skip) ? occ_ms : 0.f;  // a skip step pays for its occupancy pass
    if (cudaMemsetAsync(flag, 0, sizeof(int), stream) != cudaSuccess) {
      rc = SIMD2_ERR_CUDA;
      break;
    }
    if (step_ms) cudaEventRecord(ev[0], stream);
    const bool pk = !a_tma_ok(cur, ldcur);
    const Plan pl = make_plan(n, n, n, pk, selection_op(op));
    EpilogueArgs ep = make_epilogue(cur, ldcur, nxt, ldnxt, 1, flag, conv);
    if (use_delta) {
      if (cudaMemsetAsync(chg[par][0], 0, cmA + cmB, stream) != cudaSuccess) {
        rc = SIMD2_ERR_CUDA;
        break;
      }
      ep.chgA = chg[par][0];
      ep.chgB = chg[par][1];
      if (delta && cfg.skip) {
        ep.dA = chg[par ^ 1][0];
        ep.dB = chg[par ^ 1][1];
      }
    }
    rc = srgemm_core<float, 0>(op, n, n, n, cur, ldcur, cur, ldcur, ep, ws, pl, pk, stream, cfg);
    if (rc) break;
    if (step_ms) cudaEventRecord(ev[1], stream);
    it++;
    prev_chg = use_delta;
    par ^= 1;
    // the rules policy needs no statistics for a configuration that does not skip
    const bool next = occ_on && it < max_iter && (dispatch != 3 || config_skip(cfg_id) || step_feat);
    if (next && (rc = enqueue_occ(nxt, ldnxt))) break;
    occ_fresh = next;
    float srg_ms = 0.f;
    if ((rc = read_back(true, next))) break;
    if (step_ms) {
      cudaEventElapsedTime(&srg_ms, ev[0], ev[1]);
      step_ms[it - 1] = srg_ms + step_occ_ms;
    }
    changed = hbuf[0] != 0;
    if (next) {
      if (dispatch == 2) cfg_id = hbuf[8];
      if (step_feat && changed)
        mlp_features(n, occ.tiles_m, occ.tiles_n, occ.ktiles, hst, sms, step_feat + (size_t)it * kMlpFeat);
      settle();
    }
    std::swap(cur, nxt);
    std::swap(ldcur, ldnxt);
  }
  if (step_ms)
    for (auto& e : ev) cudaEventDestroy(e);
  if (rc) return rc;
  if (cur != X) {
    SIMD2_CUDA_TRY(cudaMemcpy2DAsync(X, ldx * 4, cur, ldcur * 4, (size_t)n * 4, n, cudaMemcpyDeviceToDevice, stream));
  }
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  if (iters_out) *iters_out = it0 + it;
  return changed ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
}

int closure_f32(int op, int n, float* X, long long ldx, int max_iter, int conv, int* iters_out,
                cudaStream_t stream) {
  return closure_f32_ex(op, n, X, ldx, max_iter, conv, 0, 0, nullptr, iters_out, nullptr, nullptr, nullptr, stream);
}

// ---------------------------------------------------------------------------
// batched closure
// ---------------------------------------------------------------------------
struct BatchedPlan {
  int dev;
  int op;
  int count;
  int max_iter;
  int conv;
  void* mem;            // one device allocation: descriptors, maps, order, queue, buffers
  BatchGraph* d_graphs;
  BatchMaps* d_maps;
  int* d_order;
  int* d_queue;
  bool fp16;            // FP16 copies exist (max_min / min_max, change test other than APLP)
  int* d_fp16_bad;      // set by the FP16 prep when an entry is not an FP16 value
  std::vector<BatchGraph> host;
};

template <int OP, bool H2>
int launch_batched(BatchedPlan* p, cudaStream_t stream) {
  auto kern = H2 ? closure_batched_h2_kernel<(OP == SIMD2_MIN_MAX ? SIMD2_MIN_MAX : SIMD2_MAX_MIN)>
                 : closure_batched_kernel<OP>;
  const size_t smem = simt_smem_bytes(kSimtStages);
  static bool configured[64] = {};
  if (!configured[p->dev]) {
    SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured[p->dev] = true;
  }
  int sms = 0;
  SIMD2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->dev));
  const int grid = std::max(1, std::min(sms, p->count));
  kern<<<grid, kSimtThreads, smem, stream>>>(p->d_graphs, p->d_maps, p->d_order, p->count, p->d_queue, p->max_iter,
                                             p->conv, p->fp16 ? p->d_fp16_bad : nullptr);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

int batched_run(BatchedPlan* p, cudaStream_t stream) {
  SIMD2_CUDA_TRY(cudaMemsetAsync(p->d_queue, 0, sizeof(int), stream));
  dim3 pg(64, std::min(p->count, 65535));
  const int* bad = p->fp16 ? p->d_fp16_bad : nullptr;
  if (p->fp16) {
    // FP16 copies first; they flag an entry that is not an FP16 value, and the
    // FP32 prep and kernel below run only then (the FP16 kernel otherwise)
    SIMD2_CUDA_TRY(cudaMemsetAsync(p->d_fp16_bad, 0, sizeof(int), stream));
    batched_prep_h_kernel<<<pg, 256, 0, stream>>>(p->d_graphs, p->count, p->d_fp16_bad);
    count_launch();
  }
  batched_prep_kernel<<<pg, 256, 0, stream>>>(p->d_graphs, p->count, bad);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  int rc;
  switch (p->op) {
    case SIMD2_MIN_PLUS: rc = launch_batched<SIMD2_MIN_PLUS, false>(p, stream); break;
    case SIMD2_MAX_PLUS: rc = launch_batched<SIMD2_MAX_PLUS, false>(p, stream); break;
    case SIMD2_MAX_MIN: rc = launch_batched<SIMD2_MAX_MIN, false>(p, stream); break;
    case SIMD2_MAX_MUL: rc = launch_batched<SIMD2_MAX_MUL, false>(p, stream); break;
    case SIMD2_MIN_MUL: rc = launch_batched<SIMD2_MIN_MUL, false>(p, stream); break;
    case SIMD2_MIN_MAX: rc = launch_batched<SIMD2_MIN_MAX, false>(p, stream); break;
    default: return SIMD2_ERR_UNSUPPORTED;
  }
  if (rc) return rc;
  if (p->fp16) {
    rc = p->op == SIMD2_MAX_MIN ? launch_batched<SIMD2_MAX_MIN, true>(p, stream)
                                : launch_batched<SIMD2_MIN_MAX, true>(p, stream);
    if (rc) return rc;
  }
  batched_finish_kernel<<<pg, 256, 0, stream>>>(p->d_graphs, p->count, bad);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

}  // namespace
}  // namespace simd2

using namespace simd2;

extern "C" {

const char* simd2_status_string(int status) {
  switch (status) {
    case SIMD2_OK: return "ok";
    case SIMD2_ERR_INVALID_ARG: return "invalid argument";
    case SIMD2_ERR_UNSUPPORTED: return "unsupported operation";
    case SIMD2_ERR_CUDA: return "CUDA runtime error";
    case SIMD2_ERR_ALLOC: return "workspace allocation failed";
    case SIMD2_ERR_TIMEOUT: return "device-side wait timed out";
    case SIMD2_ERR_NOT_CONVERGED: return "closure did not converge within max_iter";
    case SIMD2_ERR_NO_DEVICE: return "no sm_100 device";
    case SIMD2_ERR_SCRATCH_LIMIT: return "problem exceeds the fixed no-allocation scratch";
    default: return "unknown status";
  }
}

const char* simd2_version(void) { return "simd2-b200 0.1 sm_100a"; }

int simd2_srgemm(simd2_op op, int M, int N, int K, const float* A, int lda, const float* B, int ldb, const float* C,
                 int ldc, float* D, int ldd, int do_epilogue, cudaStream_t stream) {
  if (!is_float_op(op)) return op == SIMD2_OR_AND ? SIMD2_ERR_UNSUPPORTED : SIMD2_ERR_INVALID_ARG;
  int rc = check_dims(M, N, K, lda, ldb, ldc, ldd, A, B, C, D, do_epilogue);
  if (rc || M == 0 || N == 0) return rc;
  if ((rc = check_device())) return rc;
  return srgemm_f32_ws(op, M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, nullptr, 0, nullptr, stream);
}

int simd2_srgemm_orand_i32(int M, int N, int K, const int32_t* A, int lda, const int32_t* B, int ldb, const int32_t* C,
                           int ldc, int32_t* D, int ldd, int do_epilogue, cudaStream_t stream) {
  return srgemm_orand<int32_t>(M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, stream);
}

int simd2_srgemm_orand_u8(int M, int N, int K, const uint8_t* A, int lda, const uint8_t* B, int ldb, const uint8_t* C,
                          int ldc, uint8_t* D, int ldd, int do_epilogue, cudaStream_t stream) {
  return srgemm_orand<uint8_t>(M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, stream);
}

int simd2_closure(simd2_op op, int n, float* X, int ldx, int max_iter, simd2_conv conv, int* iters_out,
                  cudaStream_t stream) {
  if (conv < SIMD2_CONV_EXACT || conv > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  return closure_f32(op, n, X, ldx, max_iter, conv, iters_out, stream);
}

int simd2_closure_orand_u8(int n, uint8_t* X, int ldx, int max_iter, int* iters_out, cudaStream_t stream) {
  if (iters_out) *iters_out = 0;
  if (n < 0 || max_iter < 0 || (n > 0 && (!X || ldx < n))) return SIMD2_ERR_INVALID_ARG;
  if (n == 0 || max_iter == 0) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  // From n = 8192 a dense INT8 step takes ~0.4 ms or more, so a sparse X is
  // first squared as CSR SpGEMM steps (see closure_sparse_opening_t); smaller
  // closures would spend more on the opening's host round trips than it saves.
  int it0 = 0;
  if (n >= kOrAndSparseMinN) {
    bool ch = true;
    if ((rc = closure_sparse_opening_u8(n, X, ldx, max_iter, &it0, &ch, stream))) return rc;
    if (!ch || it0 == max_iter) {
      if (iters_out) *iters_out = it0;
      return ch ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
    }
    max_iter -= it0;
  }
  // Workspace: [tensor-core operands][Xnew n x n bytes, without delta steps][change flag][delta maps]
  const TcPlan plan = tc_plan_u8(n, n, n);
  const bool delta = use_tc2(n, n);
  const size_t x_off = align_up(plan.total, kAlign);
  const size_t f_off = x_off + (delta ? 0 : align_up((size_t)n * n, kAlign));
  // Delta steps (with the SM-pair kernel): X is squared in place -- the
  // kernel reads its operands from the packed copies made at the start of the
  // step, and each thread reads its C bytes before writing them -- so a tile
  // whose 256 rows and 256 columns did not change in the previous step is
  // skipped and keeps its bytes (step t's products of unchanged rows and
  // columns are all in X already).  Ping-pong maps of changed tile rows and
  // columns carry that from step to step.
  const int trows = (n + kTc2BM - 1) / kTc2BM, tcols = (n + kTcBN - 1) / kTcBN;
  const size_t d_off = f_off + kAlign;
  const size_t dmap = align_up((size_t)trows + tcols, kAlign);
  void* p = nullptr;
  if ((rc = get_workspace(stream, d_off + (delta ? 2 * dmap : 0), &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  uint8_t* Xn = delta ? nullptr : ws + x_off;
  int* flag = reinterpret_cast<int*>(ws + f_off);
  uint8_t* cur = X;
  long long ldcur = ldx;
  uint8_t* nxt = delta ? X : Xn;
  long long ldnxt = delta ? ldx : n;
  int it = 0, changed = 1, par = 0;
  while (changed && it < max_iter) {
    SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), stream));
    TcDelta dl;
    if (delta) {
      uint8_t* mine = ws + d_off + par * dmap;
      SIMD2_CUDA_TRY(cudaMemsetAsync(mine, 0, (size_t)trows + tcols, stream));
      dl.chg_row = mine;
      dl.chg_col = mine + trows;
      if (it > 0) {  // the first dense step has no previous maps
        const uint8_t* prev = ws + d_off + (par ^ 1) * dmap;
        dl.need_row = prev;
        dl.need_col = prev + trows;
      }
      par ^= 1;
    }
    it++;
    rc = srgemm_tc_orand<uint8_t>(n, n, n, cur, ldcur, cur, ldcur, cur, ldcur, nxt, ldnxt, 1, flag, ws, plan, stream,
                                  dl);
    if (rc) return rc;
    int h = 0;
    SIMD2_CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
    changed = h != 0;
    std::swap(cur, nxt);
    std::swap(ldcur, ldnxt);
  }
  if (cur != X) {
    SIMD2_CUDA_TRY(cudaMemcpy2DAsync(X, ldx, cur, ldcur, (size_t)n, n, cudaMemcpyDeviceToDevice, stream));
  }
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  if (iters_out) *iters_out = it0 + it;
  return changed ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
}

int simd2_closure_panel_step(simd2_op op, int rows, int n, const void* panel, int ldp, const void* full, int ldf,
                             void* out, int ldo, simd2_conv conv, int* changed, cudaStream_t stream) {
  if (rows < 0 || n < 0 || (int)op < 0 || (int)op > 8) return SIMD2_ERR_INVALID_ARG;
  if (conv < SIMD2_CONV_EXACT || conv > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  if (rows == 0 || n == 0) return SIMD2_OK;
  if (!panel || !full || !out || !changed || ldp < n || ldf < n || ldo < n) return SIMD2_ERR_INVALID_ARG;
  if (out == panel) return SIMD2_ERR_INVALID_ARG;  // the epilogue compares out with panel
  int rc = check_device();
  if (rc) return rc;
  if (op == SIMD2_OR_AND) {
    const TcPlan plan = tc_plan_u8(rows, n, n);
    void* p = nullptr;
    if ((rc = get_workspace(stream, plan.total, &p))) return rc;
    const auto* P = static_cast<const uint8_t*>(panel);
    return srgemm_tc_orand<uint8_t>(rows, n, n, P, ldp, static_cast<const uint8_t*>(full), ldf, P, ldp,
                                    static_cast<uint8_t*>(out), ldo, 1, changed, static_cast<uint8_t*>(p), plan,
                                    stream);
  }
  const auto* P = static_cast<const float*>(panel);
  return srgemm_f32_ws(op, rows, n, n, P, ldp, static_cast<const float*>(full), ldf, P, ldp,
                       static_cast<float*>(out), ldo, 1, changed, conv, nullptr, stream);
}

int simd2_closure_pred(simd2_op op, int n, float* X, int ldx, int32_t* P, int ldp, int init_pred, int max_iter,
                       int* iters_out, cudaStream_t stream) {
  if (iters_out) *iters_out = 0;
  if ((int)op < 0 || (int)op > 8) return SIMD2_ERR_INVALID_ARG;
  if (op == SIMD2_PLUS_MUL || op == SIMD2_MINUS_SQUARE || op == SIMD2_OR_AND) return SIMD2_ERR_UNSUPPORTED;
  if (n < 0 || max_iter < 0 || (n > 0 && (!X || !P || ldx < n || ldp < n))) return SIMD2_ERR_INVALID_ARG;
  if (n == 0) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  if (init_pred) {
    pred_init_kernel<<<grid_for((long long)n * n), 256, 0, stream>>>(n, X, ldx, P, ldp, add_identity(op));
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
  }
  if (max_iter == 0) return SIMD2_OK;
  // Workspace: [X' n x n][P' n x n][X^T n x n][B' Kp/2 x 2Np][packed A n x Kp][change flag]
  const size_t nn = (size_t)n * n;
  const int Kp = round_up(n, kBK), Np = round_up(n, kBN);
  const size_t x_off = 0, p_off = align_up(nn * 4, kAlign), t_off = p_off + align_up(nn * 4, kAlign);
  const size_t b_off = t_off + align_up(nn * 4, kAlign);
  const size_t a_off = b_off + align_up((size_t)Kp * Np * 4, kAlign);
  const size_t f_off = a_off + align_up((size_t)n * Kp * 4, kAlign);
  void* w = nullptr;
  if ((rc = get_workspace(stream, f_off + kAlign, &w))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(w);
  float* bufx[2] = {X, reinterpret_cast<float*>(ws + x_off)};
  int32_t* bufp[2] = {P, reinterpret_cast<int32_t*>(ws + p_off)};
  long long ldx_[2] = {ldx, n}, ldp_[2] = {ldp, n};
  float* XT = reinterpret_cast<float*>(ws + t_off);
  float* Bp = reinterpret_cast<float*>(ws + b_off);
  float* Ap = reinterpret_cast<float*>(ws + a_off);
  int* flag = reinterpret_cast<int*>(ws + f_off);
  const int tiles = (n + kBM - 1) / kBM;
  const size_t smem = pred_smem_bytes();
  const float pad = pad_value(op);
  int cur = 0, it = 0, changed = 1;
  while (changed && it < max_iter) {
    it++;
    SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), stream));
    const int nx = cur ^ 1;
    float* Xc = bufx[cur];
    const long long ldc = ldx_[cur];
    // operands of the step: X^T for the witness search, B' = X with k pairs
    // interleaved, and A = X itself when its rows suit TMA (else a packed copy)
    transpose_f32_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, stream>>>(n, Xc, ldc, XT, n);
    count_launch();
    interleave_pairs_kernel<float, 0><<<grid_for((long long)Kp / 2 * Np / 4), 256, 0, stream>>>(Xc, ldc, n, n, Bp, Kp,
                                                                                               Np, pad);
    count_launch();
    const bool pack_a = !a_tma_ok(Xc, ldc) || (n % 4 != 0);
    const float* a_base = Xc;
    long long a_pitch = ldc;
    if (pack_a) {
      pack_rows_kernel<float, 0><<<grid_for((long long)n * Kp), 256, 0, stream>>>(Xc, ldc, n, n, Ap, Kp, pad);
      count_launch();
      a_base = Ap;
      a_pitch = Kp;
    }
    SIMD2_CUDA_TRY(cudaGetLastError());
    // 16-byte loads in the witness re-scan: X's rows and X^T's rows aligned
    const int vec4 = (reinterpret_cast<uintptr_t>(Xc) % 16 == 0) && (ldc % 4 == 0) &&
                     (reinterpret_cast<uintptr_t>(XT) % 16 == 0) && (n % 4 == 0);
    CUtensorMap mA, mB;
    if ((rc = make_map_f32(&mA, a_base, n, pack_a ? Kp : n, a_pitch, kBK, kBM, CU_TENSOR_MAP_SWIZZLE_128B, true)))
      return rc;
    if ((rc = make_map_f32(&mB, Bp, Kp / 2, 2LL * Np, 2LL * Np, 2 * kBN, kBK / 2, CU_TENSOR_MAP_SWIZZLE_NONE, false)))
      return rc;
    switch (op) {
#define SIMD2_PRED_CASE(OPV)                                                                                         \
  case OPV: {                                                                                                         \
    static bool configured[64] = {};                                                                                  \
    int dev = 0;                                                                                                      \
    SIMD2_CUDA_TRY(cudaGetDevice(&dev));                                                                              \
    if (dev >= 0 && dev < 64 && !configured[dev]) {                                                                   \
      SIMD2_CUDA_TRY(cudaFuncSetAttribute(pred_fast_kernel<OPV>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                          (int)smem));                                                                \
      configured[dev] = true;                                                                                         \
    }                                                                                                                 \
    pred_fast_kernel<OPV><<<tiles * tiles, kSimtThreads, smem, stream>>>(                                             \
        mA, mB, n, Xc, ldc, XT, n, bufp[cur], ldp_[cur], bufx[nx], ldx_[nx], bufp[nx], ldp_[nx], flag, tiles, tiles,   \
        vec4);                                                                                                         \
    break;                                                                                                            \
  }
      SIMD2_PRED_CASE(SIMD2_MIN_PLUS)
      SIMD2_PRED_CASE(SIMD2_MAX_PLUS)
      SIMD2_PRED_CASE(SIMD2_MAX_MIN)
      SIMD2_PRED_CASE(SIMD2_MAX_MUL)
      SIMD2_PRED_CASE(SIMD2_MIN_MUL)
      SIMD2_PRED_CASE(SIMD2_MIN_MAX)
#undef SIMD2_PRED_CASE
      default: return SIMD2_ERR_UNSUPPORTED;
    }
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    int h = 0;
    SIMD2_CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
    changed = h != 0;
    cur = nx;
  }
  if (cur != 0) {
    SIMD2_CUDA_TRY(cudaMemcpy2DAsync(X, (size_t)ldx * 4, bufx[1], (size_t)n * 4, (size_t)n * 4, n,
                                     cudaMemcpyDeviceToDevice, stream));
    SIMD2_CUDA_TRY(cudaMemcpy2DAsync(P, (size_t)ldp * 4, bufp[1], (size_t)n * 4, (size_t)n * 4, n,
                                     cudaMemcpyDeviceToDevice, stream));
  }
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  if (iters_out) *iters_out = it;
  return changed ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
}

}  // extern "C"

namespace simd2 {
namespace {

bool spgemm_op(int op) {
  return op == SIMD2_MIN_PLUS || op == SIMD2_MAX_PLUS || op == SIMD2_MAX_MIN || op == SIMD2_MIN_MAX ||
         op == SIMD2_PLUS_MUL;
}

constexpr int kSpSmemAccMaxN = 16384;

struct SpPlan {
  int grid;            // persistent CTAs
  size_t smem;         // bitmap bytes (COUNT and FILL past kSpSmemAccMaxN columns)
  size_t smem_count;   // COUNT up to kSpSmemAccMaxN columns: one flag byte per column
  bool smem_acc;       // FILL accumulators in shared memory
  size_t smem_fill;    // FILL: bitmap + accumulators
  size_t acc_off, cnt_off, ctr_off, flag_off, tot_off, total;
};

SpPlan sp_plan(int M, int N, size_t base) {
  SpPlan p{};
  const size_t bitmap = (size_t)sp_bitmap_words(N) * 4;
  p.smem = bitmap;
  p.smem_count = (size_t)sp_flag_bytes(N);
  // the FILL pass keeps the row's accumulators in shared memory up to 16384 columns
  p.smem_acc = N <= kSpSmemAccMaxN;
  p.smem_fill = bitmap + (p.smem_acc ? (size_t)sp_acc_words(N) * 4 : 0);
  // CTAs per SM: by the FILL pass's shared memory and by the SM's 2048 threads
  int per_sm = (int)std::max<size_t>(
      1, std::min<size_t>(std::min<size_t>(8, 2048 / kSpThreads), (200u << 10) / std::max<size_t>(p.smem_fill, 1)));
  long long g = std::min<long long>((long long)M, 148LL * per_sm);
  // the accumulator slices stay below 1 GiB
  g = std::min<long long>(g, std::max<long long>(1, (1LL << 30) / (4LL * std::max(N, 1))));
  p.grid = (int)std::max<long long>(1, g);
  size_t off = base;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  p.acc_off = take(p.smem_acc ? 16 : (size_t)p.grid * N * 4);
  p.cnt_off = take((size_t)std::max(M, 1) * 4);
  p.ctr_off = take(16);
  p.flag_off = take(16);
  p.tot_off = take(16);
  p.total = off;
  return p;
}

// keys = false (CSR FILL only): the min/max FILL keeps its bitmap, for results
// sparser than 1/32 on average (the keys-only write-out reads all N keys of a row).
template <bool COUNT, bool DENSE = false, bool SMEM = false, bool KEYS = true>
int spgemm_launch(int op, const SpArgs& args, const SpPlan& plan, cudaStream_t stream, bool keys = true) {
  if constexpr (!SMEM) {
    if (plan.smem_acc) {
      if constexpr (!COUNT && !DENSE) {
        if (!keys) return spgemm_launch<COUNT, DENSE, true, false>(op, args, plan, stream);
      }
      return spgemm_launch<COUNT, DENSE, true>(op, args, plan, stream);
    }
  }
  const size_t smem = SMEM ? (COUNT ? plan.smem_count : plan.smem_fill) : plan.smem;
  auto pick = [&](auto kern) -> int {
    if (smem > (48u << 10))
      SIMD2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<plan.grid, kSpThreads, smem, stream>>>(args);
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    return SIMD2_OK;
  };
  switch (op) {
    case SIMD2_MIN_PLUS: return pick(spgemm_rows_kernel<SIMD2_MIN_PLUS, COUNT, DENSE, SMEM, KEYS>);
    case SIMD2_MAX_PLUS: return pick(spgemm_rows_kernel<SIMD2_MAX_PLUS, COUNT, DENSE, SMEM, KEYS>);
    case SIMD2_MAX_MIN: return pick(spgemm_rows_kernel<SIMD2_MAX_MIN, COUNT, DENSE, SMEM, KEYS>);
    case SIMD2_MIN_MAX: return pick(spgemm_rows_kernel<SIMD2_MIN_MAX, COUNT, DENSE, SMEM, KEYS>);
    case SIMD2_PLUS_MUL: return pick(spgemm_rows_kernel<SIMD2_PLUS_MUL, COUNT, DENSE, SMEM>);  // ordered: no keys
    default: return SIMD2_ERR_UNSUPPORTED;
  }
}

int sp_check_args(int op, int M, int N, int K, const int* ap, const int* aj, int a_nnz, const int* bp,
                  const int* bj, int b_nnz, const int* cp, const int* cj, int c_nnz) {
  if ((int)op < 0 || op > 8) return SIMD2_ERR_INVALID_ARG;
  if (!spgemm_op(op)) return SIMD2_ERR_UNSUPPORTED;
  if (M < 0 || N < 0 || K < 0 || N > (1 << 20) || a_nnz < 0 || b_nnz < 0 || c_nnz < 0) return SIMD2_ERR_INVALID_ARG;
  if (!ap || !bp || (a_nnz > 0 && !aj) || (b_nnz > 0 && !bj)) return SIMD2_ERR_INVALID_ARG;
  if (cp && c_nnz > 0 && !cj) return SIMD2_ERR_INVALID_ARG;
  return SIMD2_OK;
}

constexpr int kSpOverflow = -1;  // internal: the result needs more than 2^31 - 1 entries

// Validates the structures, counts the result's row nonzeros, forms D's
// offsets.  On kSpOverflow, *nnz_out still holds the exact count.
int spgemm_count(int op, int M, int N, int K, const int* ap, const int* aj, int a_nnz, const int* bp, const int* bj,
                 int b_nnz, const int* cp, const int* cj, int c_nnz, int* dp, long long* nnz_out, uint8_t* ws,
                 const SpPlan& plan, cudaStream_t stream) {
  int* flag = reinterpret_cast<int*>(ws + plan.flag_off);
  SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, 8, stream));
  csr_check_kernel<<<grid_for(32LL * M), 256, 0, stream>>>(M, K, ap, aj, a_nnz, flag);
  csr_check_kernel<<<grid_for(32LL * K), 256, 0, stream>>>(K, N, bp, bj, b_nnz, flag);
  count_launch();
  count_launch();
  if (cp) {
    csr_check_kernel<<<grid_for(32LL * M), 256, 0, stream>>>(M, N, cp, cj, c_nnz, flag);
    count_launch();
  }
  SIMD2_CUDA_TRY(cudaGetLastError());
  int bad = 0;
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&bad, flag, 4, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  if (bad) return SIMD2_ERR_INVALID_ARG;
  SpArgs a{};
  a.M = M, a.N = N, a.K = K, a.a_nnz = a_nnz, a.b_nnz = b_nnz, a.c_nnz = c_nnz;
  a.ap = ap, a.aj = aj, a.bp = bp, a.bj = bj, a.cp = cp, a.cj = cj;
  a.row_nnz = reinterpret_cast<int*>(ws + plan.cnt_off);
  a.acc = reinterpret_cast<float*>(ws + plan.acc_off);
  a.next_row = reinterpret_cast<int*>(ws + plan.ctr_off);
  SIMD2_CUDA_TRY(cudaMemsetAsync(a.next_row, 0, 4, stream));
  int rc = spgemm_launch<true>(op, a, plan, stream);
  if (rc) return rc;
  long long* tot = reinterpret_cast<long long*>(ws + plan.tot_off);
  offsets_scan_kernel<<<1, 1024, 0, stream>>>(a.row_nnz, M, dp, flag + 1, tot);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  int over = 0;
  long long total = 0;
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&over, flag + 1, 4, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  *nnz_out = total;
  return over ? kSpOverflow : SIMD2_OK;
}

int spgemm_fill(int op, int M, int N, int K, const int* ap, const int* aj, const float* av, int a_nnz, const int* bp,
                const int* bj, const float* bv, int b_nnz, const int* cp, const int* cj, const float* cv, int c_nnz,
                const int* dp, int* dj, float* dv, long long d_cap, uint8_t* ws, const SpPlan& plan,
                cudaStream_t stream) {
  SpArgs a{};
  a.M = M, a.N = N, a.K = K, a.a_nnz = a_nnz, a.b_nnz = b_nnz, a.c_nnz = c_nnz, a.d_cap = d_cap;
  a.ap = ap, a.aj = aj, a.av = av, a.bp = bp, a.bj = bj, a.bv = bv, a.cp = cp, a.cj = cj, a.cv = cv;
  a.dp = dp, a.dj = dj, a.dv = dv;
  a.acc = reinterpret_cast<float*>(ws + plan.acc_off);
  a.next_row = reinterpret_cast<int*>(ws + plan.ctr_off);
  SIMD2_CUDA_TRY(cudaMemsetAsync(a.next_row, 0, 4, stream));
  // d_cap is the result's entry count (every caller sizes D from COUNT)
  const bool keys = d_cap > (long long)M * (N / 32);
  return spgemm_launch<false>(op, a, plan, stream, keys);
}

// FILL pass into a dense M x N matrix D (pitch ldd) that holds the identity.
// (A 0/1 byte matrix D gets 1 at every touched column.)
template <typename T>
int spgemm_fill_dense(int op, int M, int N, int K, const int* ap, const int* aj, const float* av, int a_nnz,
                      const int* bp, const int* bj, const float* bv, int b_nnz, const int* cp, const int* cj,
                      const float* cv, int c_nnz, T* D, long long ldd, uint8_t* ws, const SpPlan& plan,
                      cudaStream_t stream) {
  SpArgs a{};
  a.M = M, a.N = N, a.K = K, a.a_nnz = a_nnz, a.b_nnz = b_nnz, a.c_nnz = c_nnz;
  a.ap = ap, a.aj = aj, a.av = av, a.bp = bp, a.bj = bj, a.bv = bv, a.cp = cp, a.cj = cj, a.cv = cv;
  if constexpr (std::is_same<T, uint8_t>::value) a.dense_u8 = D;
  else a.dense = D;
  a.ldd = ldd;
  a.acc = reinterpret_cast<float*>(ws + plan.acc_off);
  a.next_row = reinterpret_cast<int*>(ws + plan.ctr_off);
  SIMD2_CUDA_TRY(cudaMemsetAsync(a.next_row, 0, 4, stream));
  return spgemm_launch<false, true>(op, a, plan, stream);
}

// Sparse opening of a closure: while X is sparse, square it in CSR.
// A step runs as a semiring SpGEMM when X holds at most n^2/32 entries and
// the step forms at most max_products products (sum over k of row count x
// column count).  A result with more than n^2/32 entries goes straight into
// X and ends the opening.  X (pitch ldx) is rewritten when any step ran.
// T = float: X holds values, absent = the add identity of op.  T = uint8_t:
// X is a 0/1 matrix (or_and), squared as max_min over stored 1.0 values.
// *steps: steps run; *changed: false when the last one changed nothing.
// Every step gives the dense step's bits (same contract, same result).
// stats[3] = nnz, stats[4] = *products (device), for the cost model's features.
__global__ void stats_from_csr_kernel(unsigned long long* stats, long long nnz, const unsigned long long* products) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    stats[3] = (unsigned long long)nnz;
    stats[4] = *products;
  }
}

template <typename T>
int closure_sparse_opening_t(int op, int n, T* X, long long ldx, int max_iter, const OpeningPolicy& pol, int* steps,
                             bool* changed, int* step_cfg, float* step_ms, cudaStream_t stream) {
  constexpr bool kBool = std::is_same<T, uint8_t>::value;
  *steps = 0;
  *changed = true;
  if (!spgemm_op(op) || op == SIMD2_PLUS_MUL || max_iter <= 0 || n < 2) return SIMD2_OK;
  const long long nn2 = (long long)n * n;
  const long long cap = nn2 / 32;
  if (cap < 1 || cap > 0x7fffffffLL) return SIMD2_OK;
  const float ident = add_identity(op);
  const SpPlan plan = sp_plan(n, n, 0);
  // slot 1: [spgemm plan][offsets x2][columns x2][values x2][column counts][products]
  size_t off = plan.total;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  size_t rp_off[2], cj_off[2], cv_off[2];
  for (int b = 0; b < 2; b++) {
    rp_off[b] = take((size_t)(n + 1) * 4);
    cj_off[b] = take((size_t)cap * 4);
    cv_off[b] = take((size_t)cap * 4);
  }
  const size_t cc_off = take((size_t)n * 4);
  const size_t pr_off = take(16);
  void* p = nullptr;
  int rc = get_workspace_slot(stream, 1, off, &p);
  if (rc) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  int* rp[2] = {reinterpret_cast<int*>(ws + rp_off[0]), reinterpret_cast<int*>(ws + rp_off[1])};
  int* cj[2] = {reinterpret_cast<int*>(ws + cj_off[0]), reinterpret_cast<int*>(ws + cj_off[1])};
  float* cv[2] = {reinterpret_cast<float*>(ws + cv_off[0]), reinterpret_cast<float*>(ws + cv_off[1])};
  int* colcnt = reinterpret_cast<int*>(ws + cc_off);
  unsigned long long* prod = reinterpret_cast<unsigned long long*>(ws + pr_off);
  int* counts = reinterpret_cast<int*>(ws + plan.cnt_off);
  int* flag = reinterpret_cast<int*>(ws + plan.flag_off);
  long long* tot = reinterpret_cast<long long*>(ws + plan.tot_off);
  const int rows_grid = grid_for((long long)n * 32);
  const bool learned = pol.mlp != nullptr;
  // X as a dense matrix again (ident / 0 everywhere first)
  auto clear_x = [&]() -> int {
    if constexpr (kBool) {
      SIMD2_CUDA_TRY(cudaMemset2DAsync(X, (size_t)ldx, 0, (size_t)n, (size_t)n, stream));
    } else {
      fill_kernel<float><<<grid_for(nn2), 256, 0, stream>>>(X, ldx, n, n, ident);
      count_launch();
    }
    return SIMD2_OK;
  };
  cudaEvent_t ev[2] = {};
  if (step_ms)
    for (auto& e : ev) SIMD2_CUDA_TRY(cudaEventCreate(&e));
  auto destroy_events = [&]() {
    if (step_ms)
      for (auto& e : ev) cudaEventDestroy(e);
  };
  // the first step's time includes the conversion of X to CSR
  if (step_ms) cudaEventRecord(ev[0], stream);

  // X -> CSR, when sparse enough
  SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, 12, stream));
  // flag[2]: a byte other than 0 / 1 -- the dense step rewrites it to 1 and
  // counts that as a change, which a structure-only step would not see
  if constexpr (kBool) dense_row_count_u8_kernel<<<rows_grid, 256, 0, stream>>>(n, n, X, ldx, counts, flag + 2);
  else dense_row_count_kernel<<<rows_grid, 256, 0, stream>>>(n, n, X, ldx, ident, counts);
  offsets_scan_kernel<<<1, 1024, 0, stream>>>(counts, n, rp[0], flag + 1, tot);
  count_launch();
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  long long nnz = 0;
  int non01 = 0;
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&nnz, tot, 8, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&non01, flag + 2, 4, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  if (nnz > cap || non01) {
    destroy_events();
    return SIMD2_OK;
  }
  if constexpr (kBool) dense_to_csr_u8_kernel<<<rows_grid, 256, 0, stream>>>(n, n, X, ldx, rp[0], cj[0], cv[0]);
  else dense_to_csr_kernel<<<rows_grid, 256, 0, stream>>>(n, n, X, ldx, ident, rp[0], cj[0], cv[0]);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());

  int cur = 0, it = 0;
  bool ch = true, in_x = false;  // in_x: the last step wrote X itself
  bool converted = false;        // the conversion's time went into a recorded step
  while (ch && it < max_iter) {
    SIMD2_CUDA_TRY(cudaMemsetAsync(colcnt, 0, (size_t)n * 4, stream));
    SIMD2_CUDA_TRY(cudaMemsetAsync(prod, 0, 8, stream));
    csr_col_count_kernel<<<grid_for(std::max(nnz, 1LL)), 256, 0, stream>>>(cj[cur], nnz, n, colcnt);
    csr_products_kernel<<<grid_for(n), 256, 0, stream>>>(n, rp[cur], colcnt, prod);
    count_launch();
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    unsigned long long hst[5] = {};
    if (learned) {
      // the step's statistics from the CSR copy, then the MLP's choice between
      // the sparse step and the dense configurations
      const OccPlan& o = *pol.occ;
      auto* stats = reinterpret_cast<unsigned long long*>(pol.obase + o.stats);
      SIMD2_CUDA_TRY(cudaMemsetAsync(stats, 0, 8 * sizeof(unsigned long long), stream));
      SIMD2_CUDA_TRY(cudaMemsetAsync(pol.obase + o.occ32A, 0, (size_t)o.brA * o.bcA, stream));
      csr_occupancy32_kernel<<<rows_grid, 256, 0, stream>>>(n, rp[cur], cj[cur], pol.obase + o.occ32A, o.bcA);
      occupancy_panels_kernel<<<std::min(o.ktiles, 148 * 4), 256, 0, stream>>>(
          pol.obase + o.occ32A, o.bcA, o.brA, pol.obase + o.occ32A, o.bcA, o.brA, o.tiles_m, o.tiles_n, o.ktiles,
          pol.obase + o.occA, pol.obase + o.occB, stats);
      stats_from_csr_kernel<<<1, 32, 0, stream>>>(stats, nnz, prod);
      mlp_choose_kernel<<<1, 32, 0, stream>>>(pol.mlp, stats, n, o.tiles_m, o.tiles_n, o.ktiles, pol.sms,
                                              pol.can_skip, 8, 1, pol.decision);
      for (int i = 0; i < 4; i++) count_launch();
      SIMD2_CUDA_TRY(cudaGetLastError());
      SIMD2_CUDA_TRY(cudaMemcpyAsync(hst, stats, sizeof(hst), cudaMemcpyDeviceToHost, stream));
    }
    unsigned long long hp = 0;
    int choice = kSparseConfig;
    SIMD2_CUDA_TRY(cudaMemcpyAsync(&hp, prod, 8, cudaMemcpyDeviceToHost, stream));
    if (learned) SIMD2_CUDA_TRY(cudaMemcpyAsync(&choice, pol.decision, 4, cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
    if (hp > pol.max_products || choice != kSparseConfig) break;
    if (learned && pol.step_feat)
      mlp_features(n, pol.occ->tiles_m, pol.occ->tiles_n, pol.occ->ktiles, hst, pol.sms,
                   pol.step_feat + (size_t)it * kMlpFeat);
    const int nx = cur ^ 1;
    if (step_ms && converted) cudaEventRecord(ev[0], stream);
    converted = true;
    long long nn = 0;
    rc = spgemm_count(op, n, n, n, rp[cur], cj[cur], (int)nnz, rp[cur], cj[cur], (int)nnz, rp[cur], cj[cur], (int)nnz,
                      rp[nx], &nn, ws, plan, stream);
    if (rc && rc != kSpOverflow) {
      destroy_events();
      return rc;
    }
    const bool to_x = rc == kSpOverflow || nn > cap;
    if (to_x) {
      // the result is too dense for CSR: this step writes it straight into X
      // (more entries than X had, so it changed) and the dense loop goes on
      if ((rc = clear_x())) {
        destroy_events();
        return rc;
      }
      SIMD2_CUDA_TRY(cudaGetLastError());
      rc = spgemm_fill_dense<T>(op, n, n, n, rp[cur], cj[cur], cv[cur], (int)nnz, rp[cur], cj[cur], cv[cur],
                                (int)nnz, rp[cur], cj[cur], cv[cur], (int)nnz, X, ldx, ws, plan, stream);
      if (rc) {
        destroy_events();
        return rc;
      }
      in_x = true;
      ch = true;
    } else {
      rc = spgemm_fill(op, n, n, n, rp[cur], cj[cur], cv[cur], (int)nnz, rp[cur], cj[cur], cv[cur], (int)nnz, rp[cur],
                       cj[cur], cv[cur], (int)nnz, rp[nx], cj[nx], cv[nx], nn, ws, plan, stream);
      if (rc) {
        destroy_events();
        return rc;
      }
      // X' holds X's structure (C = X) plus new entries: equal counts mean equal structure
      if (nn != nnz) {
        ch = true;
      } else {
        SIMD2_CUDA_TRY(cudaMemsetAsync(flag + 2, 0, 4, stream));
        values_differ_kernel<<<grid_for(std::max(nn, 1LL)), 256, 0, stream>>>(cv[cur], cv[nx], nn, flag + 2);
        count_launch();
        SIMD2_CUDA_TRY(cudaGetLastError());
        int h = 0;
        SIMD2_CUDA_TRY(cudaMemcpyAsync(&h, flag + 2, 4, cudaMemcpyDeviceToHost, stream));
        SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
        ch = h != 0;
      }
    }
    if (step_ms) {
      cudaEventRecord(ev[1], stream);
      cudaEventSynchronize(ev[1]);
      cudaEventElapsedTime(&step_ms[it], ev[0], ev[1]);
    }
    if (step_cfg) step_cfg[it] = kSparseConfig;
    it++;
    if (to_x) break;
    cur = nx;
    nnz = nn;
  }
  destroy_events();
  if (it > 0 && !in_x) {
    if ((rc = clear_x())) return rc;
    if constexpr (kBool) csr_scatter_u8_kernel<<<rows_grid, 256, 0, stream>>>(n, rp[cur], cj[cur], X, ldx);
    else csr_scatter_kernel<<<rows_grid, 256, 0, stream>>>(n, rp[cur], cj[cur], cv[cur], X, ldx);
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
  }
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  *steps = it;
  *changed = ch;
  return SIMD2_OK;
}

// The float closure's sparse opening under a policy (see OpeningPolicy).
int closure_sparse_opening(int op, int n, float* X, long long ldx, int max_iter, const OpeningPolicy& pol,
                           int* steps, bool* changed, int* step_cfg, float* step_ms, cudaStream_t stream) {
  return closure_sparse_opening_t<float>(op, n, X, ldx, max_iter, pol, steps, changed, step_cfg, step_ms, stream);
}

// The or_and closure's opening: the dense step runs on the INT8 tensor cores
// (about 1.3 P MAC/s), so a sparse step must stay under n^3/16384 products.
int closure_sparse_opening_u8(int n, uint8_t* X, long long ldx, int max_iter, int* steps, bool* changed,
                              cudaStream_t stream) {
  const unsigned long long nn2 = (unsigned long long)n * (unsigned long long)n;
  OpeningPolicy pol;
  pol.max_products = nn2 * (unsigned long long)n / 16384ull;
  return closure_sparse_opening_t<uint8_t>(SIMD2_MAX_MIN, n, X, ldx, max_iter, pol, steps, changed, nullptr, nullptr,
                                           stream);
}

}  // namespace
}  // namespace simd2

extern "C" {

int simd2_spgemm_nnz(simd2_op op, int M, int N, int K, const int* A_rowptr, const int* A_cols, int A_nnz,
                     const int* B_rowptr, const int* B_cols, int B_nnz, const int* C_rowptr, const int* C_cols,
                     int C_nnz, int* D_rowptr, long long* nnz_out, cudaStream_t stream) {
  using namespace simd2;
  if (!nnz_out || !D_rowptr) return SIMD2_ERR_INVALID_ARG;
  *nnz_out = 0;
  int rc = sp_check_args(op, M, N, K, A_rowptr, A_cols, A_nnz, B_rowptr, B_cols, B_nnz, C_rowptr, C_cols, C_nnz);
  if (rc) return rc;
  if ((rc = check_device())) return rc;
  const SpPlan plan = sp_plan(M, N, 0);
  void* p = nullptr;
  if ((rc = get_workspace(stream, plan.total, &p))) return rc;
  if (M == 0) {
    SIMD2_CUDA_TRY(cudaMemsetAsync(D_rowptr, 0, 4, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
    return SIMD2_OK;
  }
  rc = spgemm_count(op, M, N, K, A_rowptr, A_cols, A_nnz, B_rowptr, B_cols, B_nnz, C_rowptr, C_cols, C_nnz,
                    D_rowptr, nnz_out, static_cast<uint8_t*>(p), plan, stream);
  return rc == kSpOverflow ? SIMD2_ERR_SCRATCH_LIMIT : rc;  // int32 offsets cannot hold the result
}

int simd2_spgemm_compute(simd2_op op, int M, int N, int K, const int* A_rowptr, const int* A_cols,
                         const float* A_vals, int A_nnz, const int* B_rowptr, const int* B_cols, const float* B_vals,
                         int B_nnz, const int* C_rowptr, const int* C_cols, const float* C_vals, int C_nnz,
                         const int* D_rowptr, int* D_cols, float* D_vals, long long D_nnz, cudaStream_t stream) {
  using namespace simd2;
  int rc = sp_check_args(op, M, N, K, A_rowptr, A_cols, A_nnz, B_rowptr, B_cols, B_nnz, C_rowptr, C_cols, C_nnz);
  if (rc) return rc;
  if ((A_nnz > 0 && !A_vals) || (B_nnz > 0 && !B_vals) || (C_rowptr && C_nnz > 0 && !C_vals) || !D_rowptr ||
      D_nnz < 0 || (D_nnz > 0 && (!D_cols || !D_vals)))
    return SIMD2_ERR_INVALID_ARG;
  if (M == 0 || D_nnz == 0) return SIMD2_OK;
  if ((rc = check_device())) return rc;
  const SpPlan plan = sp_plan(M, N, 0);
  void* p = nullptr;
  if ((rc = get_workspace(stream, plan.total, &p))) return rc;
  return spgemm_fill(op, M, N, K, A_rowptr, A_cols, A_vals, A_nnz, B_rowptr, B_cols, B_vals, B_nnz, C_rowptr, C_cols,
                     C_vals, C_nnz, D_rowptr, D_cols, D_vals, D_nnz, static_cast<uint8_t*>(p), plan, stream);
}

int simd2_closure_sparse(simd2_op op, int n, int* rowptr, int* cols, float* vals, long long capacity,
                         long long* nnz_inout, int max_iter, int* iters_out, cudaStream_t stream) {
  using namespace simd2;
  if (iters_out) *iters_out = 0;
  if (!nnz_inout || n < 0 || max_iter < 0 || capacity < 0 || *nnz_inout < 0 || *nnz_inout > capacity ||
      capacity > 0x7fffffffLL)
    return SIMD2_ERR_INVALID_ARG;
  int rc = sp_check_args(op, n, n, n, rowptr, cols, (int)*nnz_inout, rowptr, cols, (int)*nnz_inout, rowptr, cols,
                         (int)*nnz_inout);
  if (rc) return rc;
  if (op == SIMD2_PLUS_MUL) return SIMD2_ERR_UNSUPPORTED;  // a closure needs an idempotent add
  if (n == 0 || max_iter == 0) return SIMD2_OK;
  if ((*nnz_inout > 0 && !vals) || (capacity > 0 && (!cols || !vals))) return SIMD2_ERR_INVALID_ARG;
  if ((rc = check_device())) return rc;
  // Workspace: [spgemm plan][D offsets n+1][D columns capacity][D values capacity]
  const SpPlan plan0 = sp_plan(n, n, 0);
  const size_t dp_off = plan0.total;
  const size_t dj_off = dp_off + align_up((size_t)(n + 1) * 4, kAlign);
  const size_t dv_off = dj_off + align_up((size_t)capacity * 4 + 4, kAlign);
  const size_t total = dv_off + align_up((size_t)capacity * 4 + 4, kAlign);
  void* p = nullptr;
  if ((rc = get_workspace(stream, total, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  int* dp = reinterpret_cast<int*>(ws + dp_off);
  int* dj = reinterpret_cast<int*>(ws + dj_off);
  float* dv = reinterpret_cast<float*>(ws + dv_off);
  int* flag = reinterpret_cast<int*>(ws + plan0.flag_off);
  const float ident = add_identity(op);
  long long nnz = *nnz_inout;
  int it = 0;
  bool changed = true, dense = false;
  while (changed && it < max_iter) {
    // Closures fill in: once X is denser than 1/32 (or a step would pass the
    // int32 offsets), the dense gated closure takes over from X.
    if (nnz * 32 > (long long)n * n) {
      dense = true;
      break;
    }
    long long nn = 0;
    rc = spgemm_count(op, n, n, n, rowptr, cols, (int)nnz, rowptr, cols, (int)nnz, rowptr, cols, (int)nnz, dp, &nn,
                      ws, plan0, stream);
    if (rc == kSpOverflow || (rc == SIMD2_OK && nn * 32 > (long long)n * n && nn > capacity)) {
      dense = true;
      break;
    }
    if (rc) return rc;
    if (nn > capacity) {
      *nnz_inout = nn;  // what the next step needs
      if (iters_out) *iters_out = it;
      return SIMD2_ERR_SCRATCH_LIMIT;
    }
    it++;
    rc = spgemm_fill(op, n, n, n, rowptr, cols, vals, (int)nnz, rowptr, cols, vals, (int)nnz, rowptr, cols, vals,
                     (int)nnz, dp, dj, dv, nn, ws, plan0, stream);
    if (rc) return rc;
    // X' holds X's structure plus any new entries: equal counts mean equal
    // structure, and then the values decide
    if (nn != nnz) {
      changed = true;
    } else {
      SIMD2_CUDA_TRY(cudaMemsetAsync(flag + 2, 0, 4, stream));
      values_differ_kernel<<<grid_for(nn), 256, 0, stream>>>(vals, dv, nn, flag + 2);
      count_launch();
      SIMD2_CUDA_TRY(cudaGetLastError());
      int h = 0;
      SIMD2_CUDA_TRY(cudaMemcpyAsync(&h, flag + 2, 4, cudaMemcpyDeviceToHost, stream));
      SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
      changed = h != 0;
    }
    SIMD2_CUDA_TRY(cudaMemcpyAsync(rowptr, dp, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, stream));
    if (nn > 0) {
      SIMD2_CUDA_TRY(cudaMemcpyAsync(cols, dj, (size_t)nn * 4, cudaMemcpyDeviceToDevice, stream));
      SIMD2_CUDA_TRY(cudaMemcpyAsync(vals, dv, (size_t)nn * 4, cudaMemcpyDeviceToDevice, stream));
    }
    nnz = nn;
  }
  if (dense) {
    // dense phase: X into an n x n matrix (second workspace slot), the gated
    // dense closure for the remaining steps, then back to CSR
    void* q = nullptr;
    if ((rc = get_workspace_slot(stream, 1, (size_t)n * n * 4 + 64, &q))) return rc;
    float* Xd = static_cast<float*>(q);
    fill_kernel<float><<<grid_for((long long)n * n), 256, 0, stream>>>(Xd, n, n, n, ident);
    csr_scatter_kernel<<<grid_for((long long)n * 32), 256, 0, stream>>>(n, rowptr, cols, vals, Xd, n);
    count_launch();
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    int it2 = 0;
    const int rc2 = closure_f32(op, n, Xd, n, max_iter - it, SIMD2_CONV_EXACT, &it2, stream);
    if (rc2 && rc2 != SIMD2_ERR_NOT_CONVERGED) return rc2;
    it += it2;
    changed = rc2 == SIMD2_ERR_NOT_CONVERGED;
    // the closure's workspace (slot 0) may have moved: take it again
    if ((rc = get_workspace(stream, total, &p))) return rc;
    ws = static_cast<uint8_t*>(p);
    int* counts = reinterpret_cast<int*>(ws + plan0.cnt_off);
    flag = reinterpret_cast<int*>(ws + plan0.flag_off);
    long long* tot = reinterpret_cast<long long*>(ws + plan0.tot_off);
    SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, 8, stream));
    dense_row_count_kernel<<<grid_for((long long)n * 32), 256, 0, stream>>>(n, n, Xd, n, ident, counts);
    // offsets go to the workspace first: the caller's rowptr still describes
    // X if the result does not fit
    int* dp2 = reinterpret_cast<int*>(ws + dp_off);
    offsets_scan_kernel<<<1, 1024, 0, stream>>>(counts, n, dp2, flag + 1, tot);
    count_launch();
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    long long nn = 0;
    SIMD2_CUDA_TRY(cudaMemcpyAsync(&nn, tot, 8, cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
    if (nn > capacity) {
      *nnz_inout = nn;
      if (iters_out) *iters_out = it;
      return SIMD2_ERR_SCRATCH_LIMIT;
    }
    SIMD2_CUDA_TRY(cudaMemcpyAsync(rowptr, dp2, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, stream));
    dense_to_csr_kernel<<<grid_for((long long)n * 32), 256, 0, stream>>>(n, n, Xd, n, ident, dp2, cols, vals);
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    nnz = nn;
  }
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  *nnz_inout = nnz;
  if (iters_out) *iters_out = it;
  return changed ? SIMD2_ERR_NOT_CONVERGED : SIMD2_OK;
}

int simd2_mst(int n, const float* W, int ldw, int* edges, float* weights, int* count_out, double* total_out,
              int* iters_out, cudaStream_t stream) {
  using namespace simd2;
  if (count_out) *count_out = 0;
  if (total_out) *total_out = 0.0;
  if (iters_out) *iters_out = 0;
  if (n < 0 || !count_out || (n > 1 && (!W || ldw < n || !edges || !weights))) return SIMD2_ERR_INVALID_ARG;
  if (n <= 1) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  // slot 1: [S n x n][D n x n][count]; slot 2: the candidates; the closure uses slot 0
  const size_t nn = (size_t)n * n;
  const size_t d_off = align_up(nn * 4, kAlign), c_off = d_off + align_up(nn * 4, kAlign);
  void* p = nullptr;
  if ((rc = get_workspace_slot(stream, 1, c_off + kAlign, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  float* S = reinterpret_cast<float*>(ws);
  float* D = reinterpret_cast<float*>(ws + d_off);
  int* count = reinterpret_cast<int*>(ws + c_off);
  mst_symmetrize_kernel<<<grid_for((long long)nn), 256, 0, stream>>>(n, W, ldw, S);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  SIMD2_CUDA_TRY(cudaMemcpyAsync(D, S, nn * 4, cudaMemcpyDeviceToDevice, stream));
  int it = 0;
  rc = closure_f32(SIMD2_MIN_MAX, n, D, n, 500, SIMD2_CONV_EXACT, &it, stream);
  if (rc) return rc;
  if (iters_out) *iters_out = it;
  SIMD2_CUDA_TRY(cudaMemsetAsync(count, 0, 4, stream));
  mst_candidates_kernel<true><<<grid_for((long long)nn), 256, 0, stream>>>(n, S, D, count, 0, nullptr, nullptr);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  int m = 0;
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&m, count, 4, cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  std::vector<int> uv(2 * (size_t)m + 2);
  std::vector<float> wv((size_t)m + 1);
  if (m > 0) {
    const size_t w_off = align_up((size_t)m * 8, kAlign);
    void* q = nullptr;
    if ((rc = get_workspace_slot(stream, 2, w_off + (size_t)m * 4 + kAlign, &q))) return rc;
    int* cuv = static_cast<int*>(q);
    float* cw = reinterpret_cast<float*>(static_cast<uint8_t*>(q) + w_off);
    SIMD2_CUDA_TRY(cudaMemsetAsync(count, 0, 4, stream));
    mst_candidates_kernel<false><<<grid_for((long long)nn), 256, 0, stream>>>(n, S, D, count, m, cuv, cw);
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    SIMD2_CUDA_TRY(cudaMemcpyAsync(uv.data(), cuv, (size_t)m * 8, cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaMemcpyAsync(wv.data(), cw, (size_t)m * 4, cudaMemcpyDeviceToHost, stream));
    SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  }
  // Kruskal over the candidates in (weight, u, v) order, union-find with
  // path halving and union by size
  std::vector<int> order(m);
  for (int e = 0; e < m; e++) order[e] = e;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    if (wv[a] != wv[b]) return wv[a] < wv[b];
    if (uv[2 * a] != uv[2 * b]) return uv[2 * a] < uv[2 * b];
    return uv[2 * a + 1] < uv[2 * b + 1];
  });
  std::vector<int> parent(n), size(n, 1);
  for (int v = 0; v < n; v++) parent[v] = v;
  auto find = [&](int v) {
    while (parent[v] != v) {
      parent[v] = parent[parent[v]];
      v = parent[v];
    }
    return v;
  };
  int taken = 0;
  double total = 0.0;
  for (int e : order) {
    int a = find(uv[2 * e]), b = find(uv[2 * e + 1]);
    if (a == b) continue;
    if (size[a] < size[b]) std::swap(a, b);
    parent[b] = a;
    size[a] += size[b];
    edges[2 * taken] = uv[2 * e];
    edges[2 * taken + 1] = uv[2 * e + 1];
    weights[taken] = wv[e];
    total += wv[e];
    taken++;
  }
  *count_out = taken;
  if (total_out) *total_out = total;
  return SIMD2_OK;
}

int simd2_reserve_workspace(simd2_op op, int M, int N, int K, cudaStream_t stream, size_t* bytes_out) {
  if (M < 0 || N < 0 || K < 0 || (int)op < 0 || (int)op > 8) return SIMD2_ERR_INVALID_ARG;
  const Plan plan = make_plan(M, N, K, true);
  size_t total = plan.total + 2 * align_up((size_t)M * N * 4, kAlign) + kAlign;
  void* p = nullptr;
  int rc = get_workspace(stream, total, &p);
  if (bytes_out) *bytes_out = rc ? 0 : total;
  return rc;
}

int simd2_release_workspaces(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SIMD2_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_ws_mu);
  cudaDeviceSynchronize();
  for (auto it = g_ws.begin(); it != g_ws.end();) {
    if (std::get<0>(it->first) == dev) {
      cudaFree(it->second.first);
      it = g_ws.erase(it);
    } else {
      ++it;
    }
  }
  return SIMD2_OK;
}

long long simd2_launch_count(void) { return g_launches.load(); }

int simd2_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = true;
  g_prof_used = 0;
  g_prof_ops = 0;
  for (int k = 0; k < 4; k++) g_prof_ms[k] = 0.0, g_prof_n[k] = 0, g_prof_k_ops[k] = 0;
  return SIMD2_OK;
}

int simd2_profile_result(int kind, double* kernel_ms, long long* launches, long long* ops) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (kind < 0 || kind > 3) return SIMD2_ERR_INVALID_ARG;
  if (kernel_ms) *kernel_ms = g_prof_ms[kind];
  if (launches) *launches = g_prof_n[kind];
  if (ops) *ops = g_prof_k_ops[kind];
  return SIMD2_OK;
}

int simd2_profile_end(double* kernel_ms, long long* launches, long long* ops) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = false;
  double total = 0.0;
  for (size_t i = 0; i < g_prof_used; i++) {
    if (cudaEventSynchronize(g_prof_events[i].second) != cudaSuccess) return SIMD2_ERR_CUDA;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g_prof_events[i].first, g_prof_events[i].second) != cudaSuccess)
      return SIMD2_ERR_CUDA;
    total += ms;
    const int k = g_prof_kind[i];
    g_prof_ms[k] += ms;
    g_prof_n[k] += 1;
    g_prof_k_ops[k] += g_prof_opsv[i];
  }
  if (kernel_ms) *kernel_ms = total;
  if (launches) *launches = (long long)g_prof_used;
  if (ops) *ops = g_prof_ops;
  return SIMD2_OK;
}

int simd2_selftest_timeout(unsigned int limit_us) {
  if (limit_us == 0 || limit_us > 2000000u) return SIMD2_ERR_INVALID_ARG;
  int rc = check_device();
  if (rc) return rc;
  wait_timeout_selftest_kernel<<<1, 32>>>((uint64_t)limit_us * 1000ull);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  SIMD2_CUDA_TRY(cudaDeviceSynchronize());
  return SIMD2_OK;
}

int simd2_timeout_site(void) {
  int h = 0, zero = 0;
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  if (cudaMemcpyFromSymbol(&h, g_timeout_site, sizeof(int)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(g_timeout_site, &zero, sizeof(int)) != cudaSuccess) return -1;
  return h;
}

int simd2_device_status(void) {
  if (cudaDeviceSynchronize() != cudaSuccess) return SIMD2_ERR_CUDA;
  int h = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&h, g_device_status, sizeof(int)) != cudaSuccess) return SIMD2_ERR_CUDA;
  if (cudaMemcpyToSymbol(g_device_status, &zero, sizeof(int)) != cudaSuccess) return SIMD2_ERR_CUDA;
  return h;
}

}  // extern "C"


extern "C" {

int simd2_batched_plan_create(simd2_op op, int count, float* const* X, const int* n, const int* ldx, int max_iter,
                              simd2_conv conv, simd2_batched_plan* out) {
  if (!out) return SIMD2_ERR_INVALID_ARG;
  *out = nullptr;
  if (count < 0 || max_iter < 0 || (count > 0 && (!X || !n || !ldx))) return SIMD2_ERR_INVALID_ARG;
  if (conv < SIMD2_CONV_EXACT || conv > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  if (!is_float_op(op)) return op == SIMD2_OR_AND ? SIMD2_ERR_UNSUPPORTED : SIMD2_ERR_INVALID_ARG;
  if (is_sum_op(op)) return SIMD2_ERR_UNSUPPORTED;
  for (int g = 0; g < count; g++)
    if (n[g] < 0 || (n[g] > 0 && (!X[g] || ldx[g] < n[g]))) return SIMD2_ERR_INVALID_ARG;
  int rc = check_device();
  if (rc) return rc;
  auto* p = new BatchedPlan();
  SIMD2_CUDA_TRY(cudaGetDevice(&p->dev));
  p->op = op;
  p->count = count;
  p->max_iter = max_iter;
  p->conv = conv;
  p->host.resize(count);
  // the FP16 path of the selection semirings (the APLP change test writes
  // -FLT_MAX, which is no FP16 value)
  p->fp16 = selection_op(op) && conv != SIMD2_CONV_APLP;
  // layout: [graphs][order][queue][FP16 flag] then per-graph buffers
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  const size_t g_off = take(sizeof(BatchGraph) * std::max(count, 1));
  const size_t m_off = take(sizeof(BatchMaps) * std::max(count, 1));
  const size_t o_off = take(sizeof(int) * std::max(count, 1));
  const size_t q_off = take(sizeof(int));
  const size_t f_off = take(sizeof(int));
  std::vector<size_t> buf_off(count);
  auto half_bytes = [&](const BatchGraph& G, size_t* xh, size_t* ph) {
    *xh = p->fp16 ? (size_t)G.Mp * G.Kh * 2 : 0;
    *ph = p->fp16 ? (size_t)(G.Kh / 2) * G.Np * 4 : 0;
  };
  for (int g = 0; g < count; g++) {
    BatchGraph& G = p->host[g];
    G.n = n[g];
    G.Mp = round_up(std::max(n[g], 1), kBM);
    G.Kp = round_up(std::max(n[g], 1), kBK);
    G.Np = round_up(std::max(n[g], 1), kBN);
    G.Kh = round_up(std::max(n[g], 1), kH2BK);
    G.user = X[g];
    G.ldu = ldx[g];
    const size_t xb = (size_t)G.Mp * G.Kp * 4, pb = (size_t)(G.Kp / 2) * 2 * G.Np * 4;
    size_t xh, ph;
    half_bytes(G, &xh, &ph);
    buf_off[g] = take(2 * xb + 2 * pb);
    if (p->fp16) take(2 * xh + 2 * ph);
  }
  void* mem = nullptr;
  if (cudaMalloc(&mem, std::max(off, (size_t)kAlign)) != cudaSuccess) {
    cudaGetLastError();
    delete p;
    return SIMD2_ERR_ALLOC;
  }
  p->mem = mem;
  uint8_t* base = static_cast<uint8_t*>(mem);
  p->d_graphs = reinterpret_cast<BatchGraph*>(base + g_off);
  p->d_maps = reinterpret_cast<BatchMaps*>(base + m_off);
  p->d_order = reinterpret_cast<int*>(base + o_off);
  p->d_queue = reinterpret_cast<int*>(base + q_off);
  p->d_fp16_bad = reinterpret_cast<int*>(base + f_off);
  for (int g = 0; g < count; g++) {
    BatchGraph& G = p->host[g];
    const size_t xb = (size_t)G.Mp * G.Kp * 4, pb = (size_t)(G.Kp / 2) * 2 * G.Np * 4;
    uint8_t* b = base + buf_off[g];
    G.X[0] = reinterpret_cast<float*>(b);
    G.X[1] = reinterpret_cast<float*>(b + xb);
    G.P[0] = reinterpret_cast<float*>(b + 2 * xb);
    G.P[1] = reinterpret_cast<float*>(b + 2 * xb + pb);
    G.Xh[0] = G.Xh[1] = nullptr;
    G.Ph[0] = G.Ph[1] = nullptr;
    if (p->fp16) {
      size_t xh, ph;
      half_bytes(G, &xh, &ph);
      uint8_t* h = b + align_up(2 * xb + 2 * pb, kAlign);
      G.Xh[0] = reinterpret_cast<__half*>(h);
      G.Xh[1] = reinterpret_cast<__half*>(h + xh);
      G.Ph[0] = reinterpret_cast<uint32_t*>(h + 2 * xh);
      G.Ph[1] = reinterpret_cast<uint32_t*>(h + 2 * xh + ph);
    }
    G.iters = 0;
    G.changed = 0;
  }
  // tensor maps: A role = X[b] [Mp][Kp], B role = P[b] [Kp/2][2Np] (all padded, never out of bounds)
  std::vector<BatchMaps> hmaps(count);
  for (int g = 0; g < count; g++) {
    BatchGraph& G = p->host[g];
    for (int b = 0; b < 2 && rc == SIMD2_OK; b++) {
      rc = make_map_f32(&hmaps[g].a[b], G.X[b], G.Mp, G.Kp, G.Kp, kBK, kBM, CU_TENSOR_MAP_SWIZZLE_128B, false);
      if (rc == SIMD2_OK)
        rc = make_map_f32(&hmaps[g].b[b], G.P[b], G.Kp / 2, 2LL * G.Np, 2LL * G.Np, 2 * kBN, kBK / 2,
                          CU_TENSOR_MAP_SWIZZLE_NONE, false);
      if (p->fp16 && rc == SIMD2_OK)
        rc = make_map_2d(&hmaps[g].ah[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, G.Xh[b], G.Mp, G.Kh, G.Kh, kH2BK, kBM,
                         CU_TENSOR_MAP_SWIZZLE_128B);
      if (p->fp16 && rc == SIMD2_OK)
        rc = make_map_2d(&hmaps[g].bh[b], CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, G.Ph[b], G.Kh / 2, G.Np, G.Np, kBN,
                         kH2BK / 2, CU_TENSOR_MAP_SWIZZLE_NONE);
    }
  }
  if (rc == SIMD2_OK && count > 0 &&
      cudaMemcpy(p->d_maps, hmaps.data(), sizeof(BatchMaps) * count, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = SIMD2_ERR_CUDA;
  if (rc) {
    cudaFree(mem);
    delete p;
    return rc;
  }
  // longest-processing-time order: largest graphs first
  std::vector<int> order(count);
  for (int g = 0; g < count; g++) order[g] = g;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
  if (count > 0) {
    if (cudaMemcpy(p->d_graphs, p->host.data(), sizeof(BatchGraph) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_order, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(mem);
      delete p;
      return SIMD2_ERR_CUDA;
    }
  }
  *out = reinterpret_cast<simd2_batched_plan>(p);
  return SIMD2_OK;
}

int simd2_batched_plan_run(simd2_batched_plan plan, cudaStream_t stream) {
  auto* p = reinterpret_cast<BatchedPlan*>(plan);
  if (!p) return SIMD2_ERR_INVALID_ARG;
  if (p->count == 0 || p->max_iter == 0) return SIMD2_OK;
  return batched_run(p, stream);
}

int simd2_batched_plan_iters(simd2_batched_plan plan, int* iters_out, int* not_converged_out) {
  auto* p = reinterpret_cast<BatchedPlan*>(plan);
  if (!p) return SIMD2_ERR_INVALID_ARG;
  if (p->count == 0) {
    if (not_converged_out) *not_converged_out = 0;
    return SIMD2_OK;
  }
  std::vector<BatchGraph> h(p->count);
  SIMD2_CUDA_TRY(cudaMemcpy(h.data(), p->d_graphs, sizeof(BatchGraph) * p->count, cudaMemcpyDeviceToHost));
  int nc = 0;
  for (int g = 0; g < p->count; g++) {
    if (iters_out) iters_out[g] = h[g].iters;
    nc += h[g].changed != 0;
  }
  if (not_converged_out) *not_converged_out = nc;
  return SIMD2_OK;
}

int simd2_batched_plan_destroy(simd2_batched_plan plan) {
  auto* p = reinterpret_cast<BatchedPlan*>(plan);
  if (!p) return SIMD2_OK;
  cudaFree(p->mem);
  delete p;
  return SIMD2_OK;
}

int simd2_closure_batched(simd2_op op, int count, float* const* X, const int* n, const int* ldx, int max_iter,
                          simd2_conv conv, int* iters_out, cudaStream_t stream) {
  simd2_batched_plan plan = nullptr;
  int rc = simd2_batched_plan_create(op, count, X, n, ldx, max_iter, conv, &plan);
  if (rc) return rc;
  rc = simd2_batched_plan_run(plan, stream);
  if (!rc && cudaStreamSynchronize(stream) != cudaSuccess) rc = SIMD2_ERR_CUDA;
  int nc = 0;
  if (!rc) rc = simd2_batched_plan_iters(plan, iters_out, &nc);
  simd2_batched_plan_destroy(plan);
  if (!rc && nc > 0) rc = SIMD2_ERR_NOT_CONVERGED;
  return rc;
}

}  // extern "C"


extern "C" {

int simd2_srgemm_tuned(simd2_op op, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                       const float* C, int ldc, float* D, int ldd, int do_epilogue, int config, cudaStream_t stream) {
  if (!is_float_op(op) || is_sum_op(op)) return op == SIMD2_OR_AND || is_sum_op(op) ? SIMD2_ERR_UNSUPPORTED
                                                                                     : SIMD2_ERR_INVALID_ARG;
  if (config < 0 || config >= kNumConfigs) return SIMD2_ERR_INVALID_ARG;
  int rc = check_dims(M, N, K, lda, ldb, ldc, ldd, A, B, C, D, do_epilogue);
  if (rc || M == 0 || N == 0) return rc;
  if ((rc = check_device())) return rc;
  if (K == 0) return srgemm_k0(op, M, N, C, ldc, D, ldd, do_epilogue, stream);
  const bool pack_a = !a_tma_ok(A, lda);
  const Plan plan = make_plan(M, N, K, pack_a);
  const bool skip = config_skip(config) && skip_supported(op) && (K + kBK - 1) / kBK <= kMaxSkipKtiles;
  const OccPlan occ = make_occ_plan(M, N, K, false);
  const size_t o_off = align_up(plan.total, kAlign);
  void* p = nullptr;
  if ((rc = get_workspace(stream, o_off + (skip ? occ.total : 0), &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  SimtConfig cfg;
  cfg.split = config_split(config);
  if (skip) {
    if ((rc = compute_occupancy(op, M, N, K, A, lda, B, ldb, false, ws + o_off, occ, stream))) return rc;
    cfg.skip = true;
    cfg.occA = ws + o_off + occ.occA;
    cfg.occB = ws + o_off + occ.occB;
  }
  const EpilogueArgs ep = make_epilogue(C, ldc, D, ldd, do_epilogue, nullptr, 0);
  return srgemm_core<float, 0>(op, M, N, K, A, lda, B, ldb, ep, ws, plan, pack_a, stream, cfg);
}

int simd2_closure_ex(simd2_op op, int n, float* X, int ldx, int max_iter, simd2_conv conv, simd2_dispatch dispatch,
                     int fixed_config, const float* mlp_params, int* iters_out, int* step_configs, float* step_ms,
                     float* step_features, cudaStream_t stream) {
  if (conv < SIMD2_CONV_EXACT || conv > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  return closure_f32_ex(op, n, X, ldx, max_iter, conv, (int)dispatch, fixed_config, mlp_params, iters_out,
                        step_configs, step_ms, step_features, stream);
}

int simd2_set_dense_configs(const int* n_min, const int* config, int count) {
  if (count < 0 || (count > 0 && (!n_min || !config))) return SIMD2_ERR_INVALID_ARG;
  for (int i = 0; i < count; i++) {
    if (n_min[i] < 1 || config[i] < 0 || config[i] > 3 || (i > 0 && n_min[i] <= n_min[i - 1]))
      return SIMD2_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(g_dense_mu);
  g_dense_n.assign(n_min, n_min + count);
  g_dense_split.resize(count);
  for (int i = 0; i < count; i++) g_dense_split[i] = config_split(config[i]);
  return SIMD2_OK;
}

int simd2_mlp_param_count(void) { return kMlpParams; }

int simd2_mlp_forward(const float* params, const float* X, int batch, float* out, cudaStream_t stream) {
  if (!params || !X || !out || batch < 0) return SIMD2_ERR_INVALID_ARG;
  if (batch == 0) return SIMD2_OK;
  mlp_forward_kernel<<<grid_for(batch, 128), 128, 0, stream>>>(params, X, batch, out);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

int simd2_mlp_gradient(const float* params, const float* X, const float* y, int batch, float* grad,
                       float* sample_grads, cudaStream_t stream) {
  if (!params || !X || !y || !grad || !sample_grads || batch <= 0) return SIMD2_ERR_INVALID_ARG;
  mlp_sample_grad_kernel<<<grid_for(batch, 64), 64, 0, stream>>>(params, X, y, batch, sample_grads);
  count_launch();
  column_sum_kernel<<<grid_for(kMlpParams, 128), 128, 0, stream>>>(sample_grads, batch, kMlpParams, grad);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

int simd2_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int step, cudaStream_t stream) {
  if (!params || !grad || !m || !v || step < 1) return SIMD2_ERR_INVALID_ARG;
  adam_kernel<<<grid_for(kMlpParams, 256), 256, 0, stream>>>(params, grad, m, v, kMlpParams, lr, 0.9f, 0.999f, 1e-8f,
                                                             step);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

}  // extern "C"


// ---------------------------------------------------------------------------
// k nearest neighbours (PLD): minus_square on the tensor cores per query
// chunk, then a warp-per-row top-k with sqrt.
// ---------------------------------------------------------------------------
namespace simd2 {
namespace {

template <int KT>
int knn_topk_launch(const float* dist, long long ldd, int rows, int cols, float* od, int32_t* oi, long long ldo,
                    int kout, cudaStream_t stream) {
  knn_topk_kernel<KT><<<std::max(1, std::min(rows, 148 * 16)), kKnnWarps * 32, 0, stream>>>(dist, ldd, rows, cols, 0,
                                                                                            od, oi, ldo, kout, 1);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// Reference chunks per 128 queries for the fused kernel: one CTA per
// (query block, chunk), so the grid has qblocks * chunks CTAs, one per SM at a
// time.  Minimises waves * (tiles per chunk + a fixed cost of about three
// tiles: TMEM allocation, query load, pipeline fill and drain).
int knn_fused_chunks(int qblocks, int tiles, int sms, long long max_lists) {
  int best = 1;
  double best_cost = 1e300;
  for (int c = 1; c <= tiles; c++) {
    const int tpc = (tiles + c - 1) / c;
    const int chunks = (tiles + tpc - 1) / tpc;
    if (chunks != c) continue;
    if (2LL * chunks > max_lists) break;
    const long long units = (long long)qblocks * chunks;
    const double cost = (double)((units + sms - 1) / sms) * (tpc + 3.0);
    if (cost < best_cost) {
      best_cost = cost;
      best = c;
    }
  }
  return best;
}

// One fused pass: knn_fused_kernel<KL> over every (query block, chunk) unit,
// then the per-query merge of its lists of KL into kout results (lane lists
// of KT).  flags / gate: see knn_merge_kernel.
template <int KL, int KT>
int knn_fused_pass(const CUtensorMap& mqh, const CUtensorMap& mql, const CUtensorMap& mrh, const CUtensorMap& mrl,
                   const KnnFusedArgs& args, int qblocks, float* od, int32_t* oi, long long ldo, int kout, int* flags,
                   cudaStream_t stream) {
  static bool configured[64] = {};
  int dev = 0;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return SIMD2_ERR_NO_DEVICE;
  if (!configured[dev]) {
    SIMD2_CUDA_TRY(
        cudaFuncSetAttribute(knn_fused_kernel<KL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kKfSmemBytes));
    configured[dev] = true;
  }
  // the second pass's time counts, its operations were counted by the first
  auto* ev = prof_slot(args.gate ? 0LL : 2LL * args.Q * args.R * args.D, kProfTensor);
  if (ev) cudaEventRecord(ev->first, stream);
  knn_fused_kernel<KL><<<qblocks * args.chunks, kKfThreads, kKfSmemBytes, stream>>>(mqh, mql, mrh, mrl, args);
  count_launch();
  if (ev) cudaEventRecord(ev->second, stream);
  SIMD2_CUDA_TRY(cudaGetLastError());
  const int lists = 2 * args.chunks;
  const int G = lists <= 2 ? 2 : lists <= 4 ? 4 : lists <= 8 ? 8 : lists <= 16 ? 16 : 32;
  const int grid = grid_for((long long)(args.Q + 32 / G - 1) / (32 / G) * 32);
  auto merge = G == 2 ? knn_merge_kernel<KL, KT, 2> : G == 4 ? knn_merge_kernel<KL, KT, 4>
             : G == 8 ? knn_merge_kernel<KL, KT, 8> : G == 16 ? knn_merge_kernel<KL, KT, 16>
             : knn_merge_kernel<KL, KT, 32>;
  merge<<<grid, 256, 0, stream>>>(args.part_d, args.part_i, args.Q, lists, od, oi, ldo, kout, flags, args.gate);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

// The fused k-NN in up to two passes.  For k > 8 the first pass keeps lists
// of KT / 2 per (query, chunk half) -- about half the insertion work, and
// enough unless one half of one chunk holds more than KT / 2 of a query's
// neighbours; the merge flags every query block where that may have cut a
// list short, and the second pass redoes just those blocks with lists of KT
// (its CTAs and merge rows of unflagged blocks exit at once).  Both passes
// are enqueued; the call stays asynchronous and the result is the one-pass
// result bit for bit.  Lists of 4 for k = 5..8 are cut short in most blocks
// of 128 random queries (one of the ~30 lists holding 4 of the top 8 is
// common), so those k run one pass.
template <int KT>
int knn_fused_launch(const CUtensorMap& mqh, const CUtensorMap& mql, const CUtensorMap& mrh, const CUtensorMap& mrl,
                     KnnFusedArgs a, int qblocks, float* od, int32_t* oi, long long ldo, int kout, float* pd2,
                     int32_t* pi2, unsigned* ready2, int* flags, cudaStream_t stream) {
  if constexpr (KT >= 16) {
    if (kout > KT / 2) {
      int rc = knn_fused_pass<KT / 2, KT>(mqh, mql, mrh, mrl, a, qblocks, od, oi, ldo, kout, flags, stream);
      if (rc) return rc;
      KnnFusedArgs b = a;
      b.part_d = pd2;
      b.part_i = pi2;
      b.ready = ready2;
      b.gate = flags;
      return knn_fused_pass<KT, KT>(mqh, mql, mrh, mrl, b, qblocks, od, oi, ldo, kout, nullptr, stream);
    }
  }
  return knn_fused_pass<KT, KT>(mqh, mql, mrh, mrl, a, qblocks, od, oi, ldo, kout, nullptr, stream);
}

// Query rows per chunk so that one chunk's distance block stays near 1 GiB.
int knn_chunk_rows(int Q, int R) {
  long long rows = (1LL << 30) / (4LL * std::max(R, 1));
  rows = std::max(128LL, rows / 128 * 128);
  return (int)std::min<long long>(rows, round_up(Q, 128));
}

}  // namespace
}  // namespace simd2

namespace simd2 {
namespace {

// The fused path: operand prep, one knn_fused_kernel launch over all
// (query block, reference chunk) units, and the per-query merge.
int knn_fused(const float* query, int Q, int ldq, const float* ref, int R, int ldr, int D, int k, float* out_dist,
              int32_t* out_idx, int ldo, cudaStream_t stream) {
  const int Dp = round_up(D, 8);
  const int KT = k <= 4 ? 4 : k <= 8 ? 8 : k <= 16 ? 16 : 32;
  const int qblocks = (Q + kKfBM - 1) / kKfBM;
  const int tiles = (R + kKfBN - 1) / kKfBN;
  // partial lists: at most 256 MiB of (distance, index) pairs
  const long long max_lists = std::max(2LL, (256LL << 20) / (8LL * KT * std::max(Q, 1)));
  int dev = 0, sms = 148;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  SIMD2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // A pilot chunk of a few tiles per query block when the units fill more
  // than one wave (see knn_unit_tiles); the other chunks share the rest.
  int pilot = 0;
  int main_chunks = knn_fused_chunks(qblocks, tiles, sms, max_lists);
  if (tiles >= 64 && max_lists >= 6) {
    const int mc = knn_fused_chunks(qblocks, tiles - 4, sms, max_lists - 2);
    if ((long long)qblocks * mc > sms) {
      pilot = 4;
      main_chunks = mc;
    }
  }
  const int tpc = (tiles - pilot + main_chunks - 1) / main_chunks;
  const int chunks = main_chunks + (pilot ? 1 : 0);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  const size_t qhi = take((size_t)Q * Dp * 2), qlo = take((size_t)Q * Dp * 2);
  const size_t rhi = take((size_t)R * Dp * 2), rlo = take((size_t)R * Dp * 2);
  const size_t nq = take((size_t)Q * 4), nr = take((size_t)tiles * kKfBN * 4), tm = take((size_t)tiles * 4);
  const size_t pd = take((size_t)Q * 2 * chunks * KT * 4), pi = take((size_t)Q * 2 * chunks * KT * 4);
  // the second pass's lists; then the ready flags of both passes and the
  // first pass's block flags, side by side so that the prep kernel clears them
  const size_t pd2 = take((size_t)Q * 2 * chunks * KT * 4), pi2 = take((size_t)Q * 2 * chunks * KT * 4);
  const size_t rf = take((size_t)qblocks * chunks * 4);
  const size_t rf2 = take((size_t)qblocks * chunks * 4), qf = take((size_t)qblocks * 4);
  void* p = nullptr;
  int rc = get_workspace(stream, off, &p);
  if (rc) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  auto* q_hi = reinterpret_cast<__nv_bfloat16*>(ws + qhi);
  auto* q_lo = reinterpret_cast<__nv_bfloat16*>(ws + qlo);
  auto* r_hi = reinterpret_cast<__nv_bfloat16*>(ws + rhi);
  auto* r_lo = reinterpret_cast<__nv_bfloat16*>(ws + rlo);
  float* n_q = reinterpret_cast<float*>(ws + nq);
  float* n_r = reinterpret_cast<float*>(ws + nr);
  float* t_max = reinterpret_cast<float*>(ws + tm);
  // One launch: norms, BF16 splits, per-tile largest reference norm, +inf
  // norms for the references past R (their distances never enter a list), and
  // the cleared flags.
  KnnPrepArgs pa{};
  pa.q = query;
  pa.ldq = ldq;
  pa.Q = Q;
  pa.r = ref;
  pa.ldr = ldr;
  pa.R = R;
  pa.D = D;
  pa.Dp = Dp;
  pa.q_hi = q_hi;
  pa.q_lo = q_lo;
  pa.r_hi = r_hi;
  pa.r_lo = r_lo;
  pa.n_q = n_q;
  pa.n_r = n_r;
  pa.t_max = t_max;
  pa.r_tiles = tiles;
  pa.clear = reinterpret_cast<unsigned*>(ws + rf);
  pa.clear_words = (long long)(qf + (size_t)qblocks * 4 - rf) / 4;
  knn_prep_kernel<<<tiles + (Q + kKfBN - 1) / kKfBN, kKnnPrepThreads, 0, stream>>>(pa);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  const auto BF = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const auto SW = CU_TENSOR_MAP_SWIZZLE_128B;
  CUtensorMap mqh, mql, mrh, mrl;
  if ((rc = make_map_2d(&mqh, BF, 2, q_hi, Q, Dp, Dp, 64, kKfBM, SW))) return rc;
  if ((rc = make_map_2d(&mql, BF, 2, q_lo, Q, Dp, Dp, 64, kKfBM, SW))) return rc;
  if ((rc = make_map_2d(&mrh, BF, 2, r_hi, R, Dp, Dp, 64, kKfBN, SW))) return rc;
  if ((rc = make_map_2d(&mrl, BF, 2, r_lo, R, Dp, Dp, 64, kKfBN, SW))) return rc;
  KnnFusedArgs a{};
  a.Q = Q;
  a.R = R;
  a.D = D;
  a.panels = (Dp + 63) / 64;
  a.chunks = chunks;
  a.tiles_per_chunk = tpc;
  a.pilot_tiles = pilot;
  a.num_tiles = tiles;
  a.norm_q = n_q;
  a.norm_r = n_r;
  a.tile_nrmax = t_max;
  a.q32 = query;
  a.ldq = ldq;
  a.r32 = ref;
  a.ldr = ldr;
  a.band = kMinusSquareBand;
  a.part_d = reinterpret_cast<float*>(ws + pd);
  a.part_i = reinterpret_cast<int32_t*>(ws + pi);
  a.ready = reinterpret_cast<unsigned*>(ws + rf);
  a.kout = k;
  a.gate = nullptr;
  float* p_d2 = reinterpret_cast<float*>(ws + pd2);
  int32_t* p_i2 = reinterpret_cast<int32_t*>(ws + pi2);
  unsigned* r2 = reinterpret_cast<unsigned*>(ws + rf2);
  int* flags = reinterpret_cast<int*>(ws + qf);
  switch (KT) {
    case 4:
      return knn_fused_launch<4>(mqh, mql, mrh, mrl, a, qblocks, out_dist, out_idx, ldo, k, p_d2, p_i2, r2, flags, stream);
    case 8:
      return knn_fused_launch<8>(mqh, mql, mrh, mrl, a, qblocks, out_dist, out_idx, ldo, k, p_d2, p_i2, r2, flags, stream);
    case 16:
      return knn_fused_launch<16>(mqh, mql, mrh, mrl, a, qblocks, out_dist, out_idx, ldo, k, p_d2, p_i2, r2, flags,
                                  stream);
    default:
      return knn_fused_launch<32>(mqh, mql, mrh, mrl, a, qblocks, out_dist, out_idx, ldo, k, p_d2, p_i2, r2, flags,
                                  stream);
  }
}

}  // namespace
}  // namespace simd2

extern "C" int simd2_knn(const float* query, int Q, int ldq, const float* ref, int R, int ldr, int D, int k,
                         float* out_dist, int32_t* out_idx, int ldo, cudaStream_t stream) {
  return simd2_knn_ex(query, Q, ldq, ref, R, ldr, D, k, out_dist, out_idx, ldo, SIMD2_KNN_AUTO, stream);
}

extern "C" int simd2_knn_ex(const float* query, int Q, int ldq, const float* ref, int R, int ldr, int D, int k,
                            float* out_dist, int32_t* out_idx, int ldo, int mode, cudaStream_t stream) {
  using namespace simd2;
  if (Q < 0 || R < 0 || D < 0 || k < 1 || k > kKnnMaxK || ldo < k) return SIMD2_ERR_INVALID_ARG;
  if (mode != SIMD2_KNN_AUTO && mode != SIMD2_KNN_FUSED && mode != SIMD2_KNN_MATERIALISED)
    return SIMD2_ERR_INVALID_ARG;
  if (Q == 0) return SIMD2_OK;
  if (!query || !out_dist || !out_idx || ldq < D || (R > 0 && (!ref || ldr < D)) || R > (1 << 21) || D == 0)
    return SIMD2_ERR_INVALID_ARG;
  int rc = check_device();
  if (rc) return rc;
  if (R == 0) {
    // no reference points: +inf distances, index -1
    fill_kernel<float><<<grid_for((long long)Q * k), 256, 0, stream>>>(out_dist, ldo, Q, k, __builtin_inff());
    fill_kernel<int32_t><<<grid_for((long long)Q * k), 256, 0, stream>>>(out_idx, ldo, Q, k, -1);
    count_launch();
    count_launch();
    SIMD2_CUDA_TRY(cudaGetLastError());
    return SIMD2_OK;
  }
  const int Dp = round_up(D, 8);
  const bool fused = mode == SIMD2_KNN_FUSED || (mode == SIMD2_KNN_AUTO && Dp <= 64 * kKfMaxPanels);
  if (fused && Dp > 64 * kKfMaxPanels) return SIMD2_ERR_UNSUPPORTED;
  if (fused) return knn_fused(query, Q, ldq, ref, R, ldr, D, k, out_dist, out_idx, ldo, stream);
  const int Qc = knn_chunk_rows(Q, R);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes, kAlign); return o; };
  const size_t qhi = take((size_t)Q * Dp * 2), qlo = take((size_t)Q * Dp * 2);
  const size_t rhi = take((size_t)R * Dp * 2), rlo = take((size_t)R * Dp * 2);
  const size_t nq = take((size_t)Q * 4), nr = take((size_t)R * 4);
  const size_t dch = take((size_t)Qc * R * 4);
  void* p = nullptr;
  if ((rc = get_workspace(stream, off, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  auto* q_hi = reinterpret_cast<__nv_bfloat16*>(ws + qhi);
  auto* q_lo = reinterpret_cast<__nv_bfloat16*>(ws + qlo);
  auto* r_hi = reinterpret_cast<__nv_bfloat16*>(ws + rhi);
  auto* r_lo = reinterpret_cast<__nv_bfloat16*>(ws + rlo);
  float* n_q = reinterpret_cast<float*>(ws + nq);
  float* n_r = reinterpret_cast<float*>(ws + nr);
  float* dist = reinterpret_cast<float*>(ws + dch);
  split_rows_bf16_kernel<<<grid_for((long long)Q * Dp / 8), 256, 0, stream>>>(query, ldq, Q, D, q_hi, q_lo, Dp);
  split_rows_bf16_kernel<<<grid_for((long long)R * Dp / 8), 256, 0, stream>>>(ref, ldr, R, D, r_hi, r_lo, Dp);
  row_norms_kernel<<<grid_for((long long)Q * 32), 256, 0, stream>>>(query, ldq, Q, D, n_q);
  row_norms_kernel<<<grid_for((long long)R * 32), 256, 0, stream>>>(ref, ldr, R, D, n_r);
  for (int i = 0; i < 4; i++) count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  const auto BF = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const auto SW = tc_swizzle<0>();
  constexpr int BX = tc_box_k<0>();
  CUtensorMap mb0, mb1;
  if ((rc = make_map_2d(&mb0, BF, 2, r_hi, R, Dp, Dp, BX, kTcBN, SW))) return rc;
  if ((rc = make_map_2d(&mb1, BF, 2, r_lo, R, Dp, Dp, BX, kTcBN, SW))) return rc;
  for (int q0 = 0; q0 < Q; q0 += Qc) {
    const int rows = std::min(Qc, Q - q0);
    CUtensorMap ma0, ma1;
    if ((rc = make_map_2d(&ma0, BF, 2, q_hi + (size_t)q0 * Dp, rows, Dp, Dp, BX, kTcBM, SW))) return rc;
    if ((rc = make_map_2d(&ma1, BF, 2, q_lo + (size_t)q0 * Dp, rows, Dp, Dp, BX, kTcBM, SW))) return rc;
    TcEpilogue ep{};
    ep.op = SIMD2_MINUS_SQUARE;
    ep.do_epilogue = 0;
    ep.C = dist;
    ep.ldc = R;
    ep.D = dist;
    ep.ldd = R;
    ep.norm_a = n_q + q0;
    ep.norm_b = n_r;
    ep.A32 = query + (size_t)q0 * ldq;
    ep.lda32 = ldq;
    ep.B32 = ref;
    ep.ldb32 = ldr;
    ep.b_rows = 1;
    ep.K = D;
    ep.band = kMinusSquareBand;
    if ((rc = launch_tc<0>(rows, R, D, ma0, ma1, mb0, mb1, ep, stream))) return rc;
    float* od = out_dist + (size_t)q0 * ldo;
    int32_t* oi = out_idx + (size_t)q0 * ldo;
    if (k <= 4) rc = knn_topk_launch<4>(dist, R, rows, R, od, oi, ldo, k, stream);
    else if (k <= 8) rc = knn_topk_launch<8>(dist, R, rows, R, od, oi, ldo, k, stream);
    else if (k <= 16) rc = knn_topk_launch<16>(dist, R, rows, R, od, oi, ldo, k, stream);
    else rc = knn_topk_launch<32>(dist, R, rows, R, od, oi, ldo, k, stream);
    if (rc) return rc;
  }
  return SIMD2_OK;
}


// ---------------------------------------------------------------------------
// compatibility entries: FP16-input srgemm (tensor_srgemm) and the
// convergence test (comp_update / comp_update2)
// ---------------------------------------------------------------------------
extern "C" int simd2_srgemm_f16(simd2_op op, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                                const float* C, int ldc, float* D, int ldd, int do_epilogue, cudaStream_t stream) {
  using namespace simd2;
  if ((int)op < 0 || (int)op > 8) return SIMD2_ERR_INVALID_ARG;
  int rc = check_dims(M, N, K, lda, ldb, ldc, ldd, A, B, C, D, do_epilogue);
  if (rc || M == 0 || N == 0) return rc;
  if ((rc = check_device())) return rc;
  // or_and on {0,1}: the max_min semiring on booleans (AND = min, OR = max)
  const bool boolean = op == SIMD2_OR_AND;
  const int run_op = boolean ? SIMD2_MAX_MIN : op;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(std::max(bytes, (size_t)4), kAlign); return o; };
  const size_t a_off = take((size_t)M * K * 4), b_off = take((size_t)K * N * 4);
  const size_t c_off = take(boolean && do_epilogue ? (size_t)M * N * 4 : 4);
  const size_t plan_off = off;
  const size_t need = is_sum_op(run_op) ? tc_plan_bf16(M, N, K).total : make_plan(M, N, K, false).total;
  void* p = nullptr;
  if ((rc = get_workspace(stream, plan_off + need, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  float* Af = reinterpret_cast<float*>(ws + a_off);
  float* Bf = reinterpret_cast<float*>(ws + b_off);
  const float* Cuse = C;
  long long ldc_use = ldc;
  if (K > 0) {
    if (boolean) {
      half_to_float_kernel<1><<<grid_for((long long)M * K), 256, 0, stream>>>(static_cast<const __half*>(A), lda, M, K,
                                                                              Af);
      half_to_float_kernel<1><<<grid_for((long long)K * N), 256, 0, stream>>>(static_cast<const __half*>(B), ldb, K, N,
                                                                              Bf);
    } else {
      half_to_float_kernel<0><<<grid_for((long long)M * K), 256, 0, stream>>>(static_cast<const __half*>(A), lda, M, K,
                                                                              Af);
      half_to_float_kernel<0><<<grid_for((long long)K * N), 256, 0, stream>>>(static_cast<const __half*>(B), ldb, K, N,
                                                                              Bf);
    }
    count_launch();
    count_launch();
  }
  if (boolean && do_epilogue) {
    float* Cb = reinterpret_cast<float*>(ws + c_off);
    float_bool_kernel<<<grid_for((long long)M * N), 256, 0, stream>>>(C, ldc, M, N, Cb);
    count_launch();
    Cuse = Cb;
    ldc_use = N;
  }
  SIMD2_CUDA_TRY(cudaGetLastError());
  rc = srgemm_f32_ws(run_op, M, N, K, Af, K, Bf, N, Cuse, ldc_use, D, ldd, do_epilogue, nullptr, 0, ws + plan_off,
                     stream);
  if (rc) return rc;
  if (boolean && K == 0 && !do_epilogue) {
    // or_and identity is 0, not max_min's -inf
    fill_kernel<float><<<grid_for((long long)M * N), 256, 0, stream>>>(D, ldd, M, N, 0.0f);
    count_launch();
  }
  SIMD2_CUDA_TRY(cudaGetLastError());
  return SIMD2_OK;
}

namespace simd2 {
namespace {
template <typename T>
int compare_update(T* prev, T* cur, long long n, int mode, int* changed_out, cudaStream_t stream) {
  if (!changed_out || n < 0 || (n > 0 && (!prev || !cur))) return SIMD2_ERR_INVALID_ARG;
  *changed_out = 0;
  if (n == 0) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  void* p = nullptr;
  if ((rc = get_workspace(stream, kAlign, &p))) return rc;  // stream-ordered: the flag word is free
  int* flag = static_cast<int*>(p);
  SIMD2_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), stream));
  compare_update_kernel<T><<<grid_for(n), 256, 0, stream>>>(prev, cur, n, mode, flag);
  count_launch();
  SIMD2_CUDA_TRY(cudaGetLastError());
  int h = 0;
  SIMD2_CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  SIMD2_CUDA_TRY(cudaStreamSynchronize(stream));
  *changed_out = h != 0;
  return SIMD2_OK;
}
}  // namespace
}  // namespace simd2

extern "C" int simd2_compare_update(float* prev, float* cur, int M, int N, simd2_conv mode, int* changed_out,
                                    cudaStream_t stream) {
  if (M < 0 || N < 0 || mode < SIMD2_CONV_EXACT || mode > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  return simd2::compare_update<float>(prev, cur, (long long)M * N, (int)mode, changed_out, stream);
}

extern "C" int simd2_compare_update_i32(int32_t* prev, int32_t* cur, int M, int N, int* changed_out,
                                        cudaStream_t stream) {
  if (M < 0 || N < 0) return SIMD2_ERR_INVALID_ARG;
  return simd2::compare_update<int32_t>(prev, cur, (long long)M * N, 0, changed_out, stream);
}


// Bellman-Ford form of the closure (the reference's APBF build of
// apps/apsp/emulation/apsp_emulation.cu:99-105 and apps/aplp/emulation):
// X_{t+1} = X_t (+) A0 (x) X_t with the adjacency A0 fixed.
extern "C" int simd2_closure_bf(simd2_op op, int n, const float* A0, int lda0, float* X, int ldx, int max_iter,
                                simd2_conv conv, int* iters_out, cudaStream_t stream) {
  using namespace simd2;
  if (iters_out) *iters_out = 0;
  if (n < 0 || max_iter < 0 || !is_float_op(op) || is_sum_op(op) || (n > 0 && (!X || !A0 || ldx < n || lda0 < n)))
    return SIMD2_ERR_INVALID_ARG;
  if (conv < SIMD2_CONV_EXACT || conv > SIMD2_CONV_APLP) return SIMD2_ERR_INVALID_ARG;
  if (n == 0 || max_iter == 0) return SIMD2_OK;
  int rc = check_device();
  if (rc) return rc;
  int dev = 0, sms = 148;
  SIMD2_CUDA_TRY(cudaGetDevice(&dev));
  SIMD2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const Plan plan = make_plan(n, n, n, true, selection_op(op));
  const OccPlan occ = make_occ_plan(n, n, n, true);
  const size_t x_off = align_up(plan.total, kAlign);
  const size_t f_off = x_off + align_up((size_t)n * n * 4, kAlign);
  const size_t total = f_off + align_up((size_t)(max_iter + 1) * sizeof(int), kAlign);
  void* p = nullptr;
  if ((rc = get_workspace(stream, total, &p))) return rc;
  uint8_t* ws = static_cast<uint8_t*>(p);
  return closure_gated(op, n, X, ldx, max_iter, conv, 0, false, false, false, occ, ws, x_off,
                       reinterpret_cast<int*>(ws + f_off), nullptr, iters_out, nullptr, nullptr, sms, stream, A0,
                       lda0);
}

// ---------------------------------------------------------------------------
// srgemm without allocation
//
// Some callers cannot call cudaMalloc: code that runs inside a caller-owned
// memory pool or allocator that forbids side allocations, latency-critical
// loops where an allocation may block or synchronize the device, and
// processes that have already handed out all device memory.  For them the
// min/max srgemm keeps its scratch (the interleaved copy of B, and a packed
// copy of A when A is not TMA-aligned) in this fixed device array instead of
// the per-stream workspace.  The array is part of the module image, so every
// GPU that loads the library holds SIMD2_NOALLOC_SCRATCH_BYTES until exit.
// ---------------------------------------------------------------------------
namespace simd2 {
namespace {

static __device__ __align__(256) uint8_t g_noalloc_scratch[SIMD2_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol name is only a host-side stand-in; the address a kernel may use
// comes from cudaGetSymbolAddress with the device current.  It is looked up
// on every call (cheap once the module is loaded) rather than cached, so a
// context recreated after cudaDeviceReset never sees a stale address.  Under
// lazy module loading the first lookup on a device is what places the array
// in device memory; if the device has no room left for it that shows up here
// as cudaErrorMemoryAllocation and is reported as SIMD2_ERR_ALLOC.
int noalloc_scratch(uint8_t** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? SIMD2_ERR_ALLOC : SIMD2_ERR_CUDA;
  }
  *out = static_cast<uint8_t*>(p);
  return SIMD2_OK;
}

}  // namespace
}  // namespace simd2

extern "C" int simd2_srgemm_noalloc(simd2_op op, int M, int N, int K, const float* A, int lda, const float* B,
                                    int ldb, const float* C, int ldc, float* D, int ldd, int do_epilogue,
                                    cudaStream_t stream) {
  using namespace simd2;
  if (!is_float_op(op)) return op == SIMD2_OR_AND ? SIMD2_ERR_UNSUPPORTED : SIMD2_ERR_INVALID_ARG;
  if (is_sum_op(op)) return SIMD2_ERR_UNSUPPORTED;
  int rc = check_dims(M, N, K, lda, ldb, ldc, ldd, A, B, C, D, do_epilogue);
  if (rc || M == 0 || N == 0) return rc;
  if ((rc = check_device())) return rc;
  if (K == 0) return srgemm_k0(op, M, N, C, ldc, D, ldd, do_epilogue, stream);
  const bool pack_a = !a_tma_ok(A, lda);
  const Plan plan = make_plan(M, N, K, pack_a);
  if (plan.total > (size_t)SIMD2_NOALLOC_SCRATCH_BYTES) return SIMD2_ERR_SCRATCH_LIMIT;
  uint8_t* ws = nullptr;
  if ((rc = noalloc_scratch(&ws))) return rc;
  // Every byte of the plan is written by the prep kernels before the main
  // kernel reads it, so the scratch needs no clearing between calls.
  return srgemm_f32_ws(op, M, N, K, A, lda, B, ldb, C, ldc, D, ldd, do_epilogue, nullptr, 0, ws, stream);
}
