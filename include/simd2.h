/*
 * simd2.h -- C ABI of libsimd2, a B200 (sm_100a) semiring-GEMM engine.
 *
 * Drop-in for the srgemm operator surface of escalab/SIMD2.  Every entry
 * point returns a simd2_status (0 = success).  All calls are asynchronous on
 * `stream` unless stated otherwise; callers own every buffer they pass.
 *
 * Semantics (row-major, matching mmo::host_srgemm, kernel/host_srgemm.h:17-49):
 *   D[i,j] = id (+) A[i,0](x)B[0,j] (+) ... (+) A[i,K-1](x)B[K-1,j]   then,
 *   if do_epilogue, D[i,j] = D[i,j] (+) C[i,j]
 * where id is the add-identity of the semiring (+inf for min, -inf for max,
 * 0 for plus and or).  This is host_srgemm with D pre-filled with id, and it
 * is the cuASR device contract D = (A(x)B) (+) C of kernel/srgemm.cuh:66-81.
 * D may alias C (in-place accumulation); D must not overlap A or B.
 *
 * Exactness: the six min/max semirings and or_and are bit-exact against
 * host_srgemm.  Preconditions for that: operands hold no NaN and no -0.0,
 * and for max_mul / min_mul no product is -0.0, i.e. no zero operand meets a
 * negative one (operands >= 0, as in the reference's maxrp / minrp apps,
 * always qualify).  host_srgemm keeps the first of several products that tie
 * at zero with its sign; the device folds products in another order, so
 * outside this precondition results still equal host_srgemm's in value and
 * can differ only in the sign of a zero result.
 * plus_mul and minus_square are dense contractions computed on the tensor
 * cores (BF16 hi/lo split, FP32 accumulate); their error bound is stated in
 * the library documentation and checked against an FP64 oracle.
 */
#ifndef SIMD2_H
#define SIMD2_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The nine (add, mul) pairs, numbered as escalab/SIMD2's `enum op`
 * (kernel/tensor_srgemm.cuh:18-26) so the two enums convert one-to-one. */
typedef enum simd2_op {
  SIMD2_MIN_PLUS = 0,
  SIMD2_PLUS_MUL = 1,
  SIMD2_MAX_PLUS = 2,
  SIMD2_MAX_MIN = 3,
  SIMD2_MAX_MUL = 4,
  SIMD2_MIN_MUL = 5,
  SIMD2_MIN_MAX = 6,
  SIMD2_OR_AND = 7,
  SIMD2_MINUS_SQUARE = 8
} simd2_op;

typedef enum simd2_status {
  SIMD2_OK = 0,
  SIMD2_ERR_INVALID_ARG = 1,   /* bad size, stride, op or pointer */
  SIMD2_ERR_UNSUPPORTED = 2,   /* op/type combination without a kernel */
  SIMD2_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  SIMD2_ERR_ALLOC = 4,         /* workspace allocation failed */
  SIMD2_ERR_TIMEOUT = 5,       /* a bounded device-side wait ran out */
  SIMD2_ERR_NOT_CONVERGED = 6, /* closure hit max_iter while still changing */
  SIMD2_ERR_NO_DEVICE = 7,     /* no sm_100 device visible */
  SIMD2_ERR_SCRATCH_LIMIT = 8  /* problem needs more than SIMD2_NOALLOC_SCRATCH_BYTES */
} simd2_status;

/* Convergence test used by the closure entry points. */
typedef enum simd2_conv {
  SIMD2_CONV_EXACT = 0,   /* stop when the new matrix is bitwise unchanged */
  SIMD2_CONV_TOL = 1,     /* reference float test: |old-new| > 1e-4 is a change
                             (kernel/converge.cuh:6-14; inf-inf counts as unchanged) */
  SIMD2_CONV_APLP = 2     /* APLP test: new values in (-1,1) become -FLT_MAX,
                             then any difference is a change (converge.cuh:32-43) */
} simd2_conv;

const char* simd2_status_string(int status);

/* Library version and build target, e.g. "simd2-b200 0.1 sm_100a". */
const char* simd2_version(void);

/* Float srgemm for every semiring except or_and.
 * Replaces cuasr_<op>_srsgemm (kernel/srgemm.cuh:28-626, column-major; see
 * simd2_cuasr.h for the exact-signature shims) and, for FP32 inputs, the
 * FP16 emulation entry tensor_srgemm (kernel/tensor_srgemm.cuh:197-218).
 * Row-major; lda >= K, ldb >= N, ldc >= N, ldd >= N (elements).
 * Any M, N, K >= 0.  Uses a per-(device, stream) workspace that the library
 * allocates on first use and grows as needed (see simd2_reserve_workspace). */
int simd2_srgemm(simd2_op op, int M, int N, int K,
                 const float* A, int lda, const float* B, int ldb,
                 const float* C, int ldc, float* D, int ldd,
                 int do_epilogue, cudaStream_t stream);

/* or_and on int32 0/1 (any nonzero is true), the cuASR or_and surface
 * (kernel/srgemm.cuh:442-494).  D is written as 0/1. */
int simd2_srgemm_orand_i32(int M, int N, int K,
                           const int32_t* A, int lda, const int32_t* B, int ldb,
                           const int32_t* C, int ldc, int32_t* D, int ldd,
                           int do_epilogue, cudaStream_t stream);

/* or_and on uint8 0/1 (any nonzero is true); D is written as 0/1. */
int simd2_srgemm_orand_u8(int M, int N, int K,
                          const uint8_t* A, int lda, const uint8_t* B, int ldb,
                          const uint8_t* C, int ldc, uint8_t* D, int ldd,
                          int do_epilogue, cudaStream_t stream);

/* Repeated-squaring closure X <- X (+) X(x)X on an n x n matrix, in place,
 * until the convergence test reports no change or max_iter steps ran.
 * Replaces the closure loops of apps/{apsp,aplp,mcp,maxrp,minrp,mst}
 * (e.g. apps/apsp/cuASR/apsp_cuASR.cu:37-54) together with comp_update /
 * comp_update2 (kernel/converge.cuh:16-84).  *iters_out receives the number
 * of srgemm steps, counting the final unchanged one as the reference does.
 * Synchronous: returns after the result is in X.  Returns
 * SIMD2_ERR_NOT_CONVERGED if max_iter steps ran and the last still changed. */
int simd2_closure(simd2_op op, int n, float* X, int ldx, int max_iter,
                  simd2_conv conv, int* iters_out, cudaStream_t stream);

/* Bellman-Ford form X <- X (+) A0 (x) X with the adjacency A0 fixed (the
 * reference's APBF build, apps/apsp/emulation/apsp_emulation.cu:99-105);
 * same convergence tests and step counting as simd2_closure.  Synchronous. */
int simd2_closure_bf(simd2_op op, int n, const float* A0, int lda0, float* X, int ldx, int max_iter,
                     simd2_conv conv, int* iters_out, cudaStream_t stream);

/* or_and transitive closure on uint8 0/1 (apps/gtc/cuASR), synchronous.
 * From n = 8192 a sparse X is first squared as CSR SpGEMM steps (while X
 * holds at most n^2/32 entries and a step forms at most n^3/16384 products),
 * then on the INT8 tensor cores; same result and step count either way. */
int simd2_closure_orand_u8(int n, uint8_t* X, int ldx, int max_iter,
                           int* iters_out, cudaStream_t stream);

/* Batched closure: `count` independent n[g] x n[g] matrices X[g] (device
 * pointers, row pitch ldx[g]) closed in place in ONE persistent kernel launch,
 * each graph by one CTA until its own fixed point (per-graph convergence,
 * bit-exact per graph, same iteration counts as simd2_closure).  Six min/max
 * semirings.  X, n and ldx are host arrays.
 *   plan_create  allocates the plan's device memory and uploads descriptors
 *                (synchronous);
 *   plan_run     launches prep + persistent closure + copy-back on `stream`
 *                and nothing else (no allocation, no host sync), so it can be
 *                captured in a CUDA graph and replayed;
 *   plan_iters   reads the per-graph step counts (synchronous);
 *   closure_batched = create + run + iters + destroy, synchronous; returns
 *                SIMD2_ERR_NOT_CONVERGED if any graph hit max_iter. */
typedef struct simd2_batched_plan_st* simd2_batched_plan;
int simd2_batched_plan_create(simd2_op op, int count, float* const* X, const int* n, const int* ldx, int max_iter,
                              simd2_conv conv, simd2_batched_plan* plan_out);
int simd2_batched_plan_run(simd2_batched_plan plan, cudaStream_t stream);
int simd2_batched_plan_iters(simd2_batched_plan plan, int* iters_out, int* not_converged_out);
int simd2_batched_plan_destroy(simd2_batched_plan plan);
int simd2_closure_batched(simd2_op op, int count, float* const* X, const int* n, const int* ldx, int max_iter,
                          simd2_conv conv, int* iters_out, cudaStream_t stream);

/* Kernel configurations of the CUDA-core path (min/max semirings):
 * config = s | (skip << 2), split-K factor 1 << s (s in 0..3) over a
 * thread-block cluster whose CTAs fold their partial tiles through
 * distributed shared memory, and skip = 1 to drop k-blocks whose A or B block
 * holds only the (x)-annihilator (block occupancy computed per call; applies
 * to min_plus, max_plus, max_min, min_max).  All configurations give the same
 * bits.  No reference counterpart: the autotuner and the learned dispatch
 * use it. */
int simd2_srgemm_tuned(simd2_op op, int M, int N, int K,
                       const float* A, int lda, const float* B, int ldb,
                       const float* C, int ldc, float* D, int ldd,
                       int do_epilogue, int config, cudaStream_t stream);

typedef enum simd2_dispatch {
  SIMD2_DISPATCH_DENSE = 0,   /* no block skipping; split-K chosen from the tile count
                                 (the plain autotuned dense path) */
  SIMD2_DISPATCH_FIXED = 1,   /* `fixed_config` every step (8: sparse steps, see below) */
  SIMD2_DISPATCH_LEARNED = 2, /* the MLP cost model picks each step's config, sparse or dense */
  SIMD2_DISPATCH_RULES = 3    /* the hand-written policy: sparse steps under fixed
                                 thresholds, then `fixed_config` (no MLP) */
} simd2_dispatch;

/* simd2_closure with a dispatch policy.  mlp_params: device array of
 * simd2_mlp_param_count() floats (LEARNED only).  Optional host outputs of
 * max_iter entries: step_configs (config run per step; 8 = a CSR SpGEMM
 * step), step_ms (device time of each step), step_features (9 floats per
 * step: the cost-model features).  Results are bit-identical for every
 * policy.
 *
 * LEARNED and RULES decide per step only for n > 1024: a decision (statistics
 * pass, MLP launch, host round trip) costs about as much as a whole dense
 * step below that, so smaller closures run the DENSE path (step_features then
 * stay zero).  Above that, with SIMD2_CONV_EXACT and a semiring
 * simd2_spgemm_compute supports, both open with CSR SpGEMM steps while X
 * holds at most n^2/32 entries (a result past that is written densely and
 * ends the opening):
 *   LEARNED runs a sparse step when the MLP predicts it faster than every
 *   dense configuration (steps past n^3/16 products are never sparse);
 *   RULES runs it when the step forms at most n^3/256 products.
 * The dense steps then follow the MLP's per-step choice (LEARNED) or
 * fixed_config (RULES) for n > 2048, and the DENSE path for
 * 1024 < n <= 2048.  Once every block of X is occupied no step can skip, and
 * both keep the last split factor without the statistics pass.
 * FIXED with fixed_config 8 runs sparse steps while X holds at most n^2/32
 * entries and a step forms at most n^3/16 products, then the DENSE path: the
 * autotuner records sparse-step times with it. */
int simd2_closure_ex(simd2_op op, int n, float* X, int ldx, int max_iter, simd2_conv conv,
                     simd2_dispatch dispatch, int fixed_config, const float* mlp_params,
                     int* iters_out, int* step_configs, float* step_ms, float* step_features,
                     cudaStream_t stream);

/* The plain dense path's split-K factor by size, as the autotuner measured it
 * (no reference counterpart).  Entry i (n_min ascending, config 0..3: split
 * 1 << config, no skip) applies to closures of n_min[i] <= n < n_min[i + 1];
 * below n_min[0] the dense path keeps its rule (the largest split with
 * tiles * split <= SMs, at most 4).  count = 0 clears the table.  Applies to
 * simd2_closure and to SIMD2_DISPATCH_DENSE of simd2_closure_ex in this
 * process; same bits whatever the split. */
int simd2_set_dense_configs(const int* n_min, const int* config, int count);

/* Cost-model MLP (15-32-32-1, ReLU) kernels.  X: [batch][15] features+config,
 * y: [batch] targets (log2 ms).  simd2_mlp_gradient writes d/dparams of
 * mean((f(X)-y)^2) to grad (param_count floats) using sample_grads
 * ([batch][param_count] floats) as scratch; the batch sum is deterministic.
 * simd2_mlp_adam applies one Adam step (beta 0.9/0.999, eps 1e-8), step >= 1. */
int simd2_mlp_param_count(void);
int simd2_mlp_forward(const float* params, const float* X, int batch, float* out, cudaStream_t stream);
int simd2_mlp_gradient(const float* params, const float* X, const float* y, int batch, float* grad,
                       float* sample_grads, cudaStream_t stream);
int simd2_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int step,
                   cudaStream_t stream);

/* k nearest neighbours, the PLD tail of the reference
 * (apps/pld/cuASR/knncuda.cu:479-514: minus_square srgemm, then
 * modified_insertion_sort_linear and compute_sqrt_linear).
 * query [Q][D] (pitch ldq) and ref [R][D] (pitch ldr), row-major, device.
 * Writes, per query, the k smallest Euclidean distances (sqrt of the
 * minus_square sum, ascending) and the reference indices into out_dist /
 * out_idx [Q][k] (pitch ldo) -- query-major, the transpose of the
 * reference's k x Q layout.  Equal distances keep the lower index first.
 * 1 <= k <= 32, R <= 2^21.  Squared distances come from the BF16 hi/lo
 * tensor-core path with FP64 norms and the exact FP32 recompute inside the
 * cancellation band (near-duplicate points). */
int simd2_knn(const float* query, int Q, int ldq, const float* ref, int R, int ldr, int D, int k,
              float* out_dist, int32_t* out_idx, int ldo, cudaStream_t stream);

/* Execution strategy of simd2_knn_ex.  Both give bit-identical results. */
typedef enum {
  SIMD2_KNN_AUTO = 0,         /* FUSED when D <= 128, else MATERIALISED */
  SIMD2_KNN_FUSED = 1,        /* selection inside the distance MMA's epilogue; D <= 128
                                 (SIMD2_ERR_UNSUPPORTED otherwise) */
  SIMD2_KNN_MATERIALISED = 2  /* distance blocks of ~1 GiB written, then selected */
} simd2_knn_mode;

/* simd2_knn with an explicit strategy; simd2_knn(...) is
 * simd2_knn_ex(..., SIMD2_KNN_AUTO, stream). */
int simd2_knn_ex(const float* query, int Q, int ldq, const float* ref, int R, int ldr, int D, int k,
                 float* out_dist, int32_t* out_idx, int ldo, int mode, cudaStream_t stream);

/* srgemm with FP16 A and B (row-major, __half*), FP32 C and D: the entry
 * behind tensor_srgemm (kernel/tensor_srgemm.cuh:197-218).  The halves are
 * widened to FP32 exactly and the FP32 engine runs; or_and treats any
 * nonzero as true and writes 0/1.  (The reference's FP16 emulation kernel
 * rounds each product to FP16 and starts the max semirings from 0; this
 * entry keeps FP32 products and the true identities.) */
int simd2_srgemm_f16(simd2_op op, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                     const float* C, int ldc, float* D, int ldd, int do_epilogue, cudaStream_t stream);

/* The change test of the reference's closure loop (comp_update /
 * comp_update2, kernel/converge.cuh:16-84) as one call: compares prev and
 * cur (M x N, dense) under `mode` (SIMD2_CONV_TOL = comp_update,
 * SIMD2_CONV_APLP = comp_update2, which also rewrites cur; SIMD2_CONV_EXACT =
 * bitwise), copies cur into prev and returns *changed_out = 0/1.
 * Synchronous, like the reference. */
int simd2_compare_update(float* prev, float* cur, int M, int N, simd2_conv mode, int* changed_out,
                         cudaStream_t stream);
int simd2_compare_update_i32(int32_t* prev, int32_t* cur, int M, int N, int* changed_out, cudaStream_t stream);

/* One repeated-squaring step for the rows one rank owns when an n x n
 * closure is split into row panels across GPUs (the multi-GPU form of the
 * loop in apps/apsp/cuASR/apsp_cuASR.cu:37-54):
 *   out = panel (+) panel (x) full
 * panel: this rank's `rows` rows of X (pitch ldp); full: all n rows of X
 * (pitch ldf, e.g. gathered from the ranks); out: rows x n (pitch ldo, not
 * aliasing panel).  ORs 1 into the device int *changed when any element of
 * out differs from panel (conv as in simd2_closure).  float* for the float
 * semirings, uint8_t* 0/1 for SIMD2_OR_AND.  Asynchronous on stream. */
int simd2_closure_panel_step(simd2_op op, int rows, int n, const void* panel, int ldp, const void* full, int ldf,
                             void* out, int ldo, simd2_conv conv, int* changed, cudaStream_t stream);

/* Closure with a predecessor matrix, for path reconstruction (the
 * Floyd-Warshall baselines' pred output, apps/maxrp/baseline/lib/apsp.cpp:
 * 11-25 and main.cpp:80-94).  X (n x n, pitch ldx) is closed in place as by
 * simd2_closure (exact convergence); P (int32, pitch ldp) ends with
 * P[i][j] = the vertex before j on the best i -> j path found, -1 where there
 * is none and on the diagonal.  init_pred = 1 fills P from X first (i where
 * X[i][j] is an edge, i.e. not the add identity, and i != j; else -1);
 * init_pred = 0 takes the caller's P.  Per step, an element that strictly
 * improves through the lowest such k takes P[k][j].  Semirings with a min or
 * max add (min_plus, max_plus, max_min, max_mul, min_mul, min_max). */
int simd2_closure_pred(simd2_op op, int n, float* X, int ldx, int32_t* P, int ldp, int init_pred, int max_iter,
                       int* iters_out, cudaStream_t stream);

/* Semiring SpGEMM on CSR matrices, for inputs too sparse for the dense
 * kernels -- the regime that density_verification/sp_gemm_comp.cu measures
 * with cuSPARSE SpGEMM (plus-times) against dense GEMM.
 *   D = A (x) B [(+) C],   A: M x K, B: K x N, C and D: M x N
 * An absent entry is the add identity, which must annihilate the multiply:
 * SIMD2_MIN_PLUS, SIMD2_MAX_PLUS, SIMD2_MAX_MIN, SIMD2_MIN_MAX and
 * SIMD2_PLUS_MUL (others: SIMD2_ERR_UNSUPPORTED).  CSR with int32 offsets
 * (rows + 1, starting at 0) and columns strictly increasing within a row;
 * float values.  D stores every column reached through stored entries, in
 * increasing order, with the value host_srgemm (kernel/host_srgemm.h:17-49)
 * gives the dense matrices: products combined in increasing k from the add
 * identity, then C -- bit-identical, plus_mul included.  N <= 2^20.
 *
 * Two calls, as cuSPARSE's SpGEMM: simd2_spgemm_nnz checks the structures
 * (SIMD2_ERR_INVALID_ARG for malformed CSR), writes D_rowptr (M + 1 ints)
 * and returns the entry count in *nnz_out (synchronous); the caller then
 * allocates D_cols / D_vals of that size and calls simd2_spgemm_compute with
 * the same A, B, C (asynchronous).  C_rowptr = NULL: no C term. */
int simd2_spgemm_nnz(simd2_op op, int M, int N, int K, const int* A_rowptr, const int* A_cols, int A_nnz,
                     const int* B_rowptr, const int* B_cols, int B_nnz, const int* C_rowptr, const int* C_cols,
                     int C_nnz, int* D_rowptr, long long* nnz_out, cudaStream_t stream);
int simd2_spgemm_compute(simd2_op op, int M, int N, int K, const int* A_rowptr, const int* A_cols,
                         const float* A_vals, int A_nnz, const int* B_rowptr, const int* B_cols, const float* B_vals,
                         int B_nnz, const int* C_rowptr, const int* C_cols, const float* C_vals, int C_nnz,
                         const int* D_rowptr, int* D_cols, float* D_vals, long long D_nnz, cudaStream_t stream);

/* Closure X <- X (+) X (x) X of an n x n CSR matrix, in place, until
 * unchanged (the loop of apps/apsp/cuASR/apsp_cuASR.cu:37-54 on sparse
 * storage; exact convergence).  cols / vals hold `capacity` entries, the
 * first *nnz_inout of them in use; on return *nnz_inout is the closed
 * matrix's count.  When a step needs more than `capacity` entries the call
 * returns SIMD2_ERR_SCRATCH_LIMIT with X as of the previous step and the
 * needed count in *nnz_inout.  Semirings as simd2_spgemm_nnz. */
int simd2_closure_sparse(simd2_op op, int n, int* rowptr, int* cols, float* vals, long long capacity,
                         long long* nnz_inout, int max_iter, int* iters_out, cudaStream_t stream);

/* Minimum spanning forest of an undirected weighted graph from its minimax
 * closure.  The reference's mst app (apps/mst/cuASR/mst_cuASR.cu) computes
 * the min_max closure D[u][v] = min over u-v paths of the largest edge
 * weight; an edge belongs to the spanning forest that Kruskal builds in
 * (weight, u, v) order exactly when it is chosen from the edges with
 * w(u, v) == D[u][v], which this entry scans for on the GPU before a
 * union-find on the host.
 * W: n x n device matrix (pitch ldw), +inf where there is no edge; the
 * undirected weight of {u, v} is min(W[u][v], W[v][u]); the diagonal is
 * ignored.  Outputs in HOST memory: edges[2e], edges[2e+1] (u < v) and
 * weights[e] for e < *count_out (at most n - 1; fewer when the graph is
 * disconnected), in Kruskal order; *total_out the weight sum (FP64);
 * *iters_out the closure's step count.  Synchronous. */
int simd2_mst(int n, const float* W, int ldw, int* edges, float* weights, int* count_out, double* total_out,
              int* iters_out, cudaStream_t stream);

/* Reserve the per-(device, stream) workspace for srgemm calls up to
 * M x N x K so that later calls (e.g. inside stream capture) allocate
 * nothing.  Returns the bytes now reserved in *bytes_out (may be NULL). */
int simd2_reserve_workspace(simd2_op op, int M, int N, int K, cudaStream_t stream,
                            size_t* bytes_out);

/* Free every workspace the library holds on the current device. */
int simd2_release_workspaces(void);

/* Running total of kernels this library has launched in this process. */
long long simd2_launch_count(void);

/* Kernel timing: between begin and end, every main srgemm kernel launch is
 * bracketed by CUDA events on its own stream.  end() waits for them and
 * returns the summed kernel time, the number of timed launches and the
 * algorithmic operation count (2*M*N*K per launch). */
int simd2_profile_begin(void);
int simd2_profile_end(double* kernel_ms, long long* launches, long long* ops);
/* After simd2_profile_end: the same totals for one kernel family
 * (0 = CUDA-core srgemm, 1 = tensor-core srgemm). */
int simd2_profile_result(int kind, double* kernel_ms, long long* launches, long long* ops);

/* Failure-detection self-test: one kernel waits, for at most limit_us
 * microseconds (<= 2 s), on a barrier that nothing completes, then records
 * SIMD2_ERR_TIMEOUT (wait site 99) in the device error word exactly as a
 * real lost arrival would.  Synchronous; afterwards simd2_device_status()
 * returns SIMD2_ERR_TIMEOUT and the device stays usable.  No counterpart in
 * the reference. */
int simd2_selftest_timeout(unsigned int limit_us);

/* Read and clear the id of the last bounded wait that ran out (0 = none);
 * a diagnostic companion of simd2_device_status(). */
int simd2_timeout_site(void);

/* Read and clear the device-side error word that kernels set when a bounded
 * wait runs out (SIMD2_ERR_TIMEOUT).  Synchronizes the current device. */
int simd2_device_status(void);

/* Size of the fixed device scratch used by simd2_srgemm_noalloc (16 MiB).
 * Every GPU that loads libsimd2 holds this much device memory until exit. */
#define SIMD2_NOALLOC_SCRATCH_BYTES (16u << 20)

/* simd2_srgemm for the six min/max semirings (min_plus, max_plus, max_min,
 * max_mul, min_mul, min_max) that allocates nothing.  No counterpart in the
 * reference: it is for callers that must not call cudaMalloc -- code running
 * under a caller-owned memory pool or allocator that forbids side
 * allocations, real-time loops where an allocation may block, and processes
 * that have already placed all device memory.  Same arguments and results
 * as simd2_srgemm.
 *
 * Its working copy of B (k-pair interleaved, padded) and, when A's rows are
 * not 16-byte aligned, a packed copy of A live in one file-scope device
 * array of SIMD2_NOALLOC_SCRATCH_BYTES, so roundup(K,32) * roundup(N,128) * 4
 * bytes (+ M * roundup(K,32) * 4 when A is repacked) must fit in it;
 * larger problems return SIMD2_ERR_SCRATCH_LIMIT.  The other five semirings
 * return SIMD2_ERR_UNSUPPORTED.
 *
 * Each call looks up that array's device address (cudaGetSymbolAddress)
 * with the device current.  With CUDA's lazy module loading the array is
 * only placed in device memory by the first call on a device, so a caller
 * that is going to hand out all device memory makes one small call first
 * (and makes that first call before any stream capture); if the device has
 * no room left for the array, the call returns SIMD2_ERR_ALLOC.  Every
 * call, on every stream, shares the one array and
 * each call overwrites the part it uses completely before reading it (nothing
 * has to start at zero), so calls whose kernels can overlap on the GPU race
 * with each other: order them on one stream or synchronize between them. */
int simd2_srgemm_noalloc(simd2_op op, int M, int N, int K,
                         const float* A, int lda, const float* B, int ldb,
                         const float* C, int ldc, float* D, int ldd,
                         int do_epilogue, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* SIMD2_H */
