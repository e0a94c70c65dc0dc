/*
 * simd2_oracle.c -- CPU restatement of the SIMD2 srgemm contract.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked only by
 * the test-suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg.  The product library (libsimd2) never links or calls it.
 *
 * What it restates (reference paths are relative to the escalab/SIMD2 tree):
 *   - mmo::host_srgemm<T>          kernel/host_srgemm.h:17-49
 *       D[i,j] = addop(D[i,j], mulop(A[i,k], B[k,j])) for k = 0..K-1 in order,
 *       then, if do_epilogue, D[i,j] = addop(D[i,j], C[i,j]).  Row-major,
 *       lda/ldb/ldc ignored (the reference indexes A[i*K+k], B[k*N+j]).
 *   - the operator functors        kernel/host_srgemm.h:53-85
 *       minimum = std::min(lhs,rhs) = (rhs < lhs) ? rhs : lhs
 *       maximum = std::max(lhs,rhs) = (lhs < rhs) ? rhs : lhs
 *       minussquare = (lhs-rhs)*(lhs-rhs), bin_and = lhs && rhs, bin_or = lhs || rhs
 *   - the nine (add, mul) pairs    kernel/tensor_srgemm.cuh:18-26 (enum op)
 *   - repeated-squaring closure    apps/apsp/cuASR/apsp_cuASR.cu:42-54 with the
 *       change test of kernel/converge.cuh:6-14 (float), :61-69 (int) and
 *       the APLP variant :32-43.
 *   - closure with predecessors    apps/maxrp/baseline/lib/apsp.cpp:11-25 (pred
 *       rule), restated for repeated squaring (oracle_closure_pred_f32).
 *   - k-NN selection               apps/pld/baseline/test.cpp:132-182 (knn_c) with
 *       the modified insertion sort of apps/pld/emulation/knncuda.cu:171-221
 *       (ties keep the lower reference index).
 *
 * The loop order here is i-k-j instead of the reference's i-j-k.  For every
 * output element the k terms are still combined one at a time in increasing
 * k, so each element sees the identical sequence of rounded operations and the
 * result is bit-identical (compile with -ffp-contract=off so that a*b+c is not
 * fused).  The reordering only makes the B access unit-stride.
 *
 * Rows are split into panels across POSIX threads; each panel is the same
 * sequential computation on its rows, so threading does not change results.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum {
  OP_MIN_PLUS = 0,
  OP_PLUS_MUL = 1,
  OP_MAX_PLUS = 2,
  OP_MAX_MIN = 3,
  OP_MAX_MUL = 4,
  OP_MIN_MUL = 5,
  OP_MIN_MAX = 6,
  OP_OR_AND = 7,
  OP_MINUS_SQUARE = 8
};

/* std::min / std::max exactly as libstdc++ defines them (accumulator first). */
static inline float s_min(float lhs, float rhs) { return (rhs < lhs) ? rhs : lhs; }
static inline float s_max(float lhs, float rhs) { return (lhs < rhs) ? rhs : lhs; }

static inline float f_add(int op, float d, float p) {
  switch (op) {
    case OP_MIN_PLUS: case OP_MIN_MUL: case OP_MIN_MAX: return s_min(d, p);
    case OP_MAX_PLUS: case OP_MAX_MIN: case OP_MAX_MUL: return s_max(d, p);
    default: return d + p; /* plus_mul, minus_square */
  }
}

/* ------------------------------------------------------------------ */
/* float srgemm, one row panel                                          */
/* ------------------------------------------------------------------ */
#define PANEL_LOOP(MULEXPR, ADDEXPR)                                   \
  for (int i = r0; i < r1; i++) {                                      \
    float* d = D + (size_t)i * N;                                      \
    const float* a = A + (size_t)i * K;                                \
    for (int k = 0; k < K; k++) {                                      \
      const float av = a[k];                                           \
      const float* b = B + (size_t)k * N;                              \
      for (int j = 0; j < N; j++) {                                    \
        const float bv = b[j];                                         \
        const float p = (MULEXPR);                                     \
        const float dv = d[j];                                         \
        d[j] = (ADDEXPR);                                              \
      }                                                                \
    }                                                                  \
  }

static void srgemm_f32_rows(int op, int r0, int r1, int N, int K, const float* A, const float* B,
                            const float* C, float* D, int do_epilogue) {
  switch (op) {
    case OP_MIN_PLUS: PANEL_LOOP(av + bv, (p < dv) ? p : dv); break;
    case OP_PLUS_MUL: PANEL_LOOP(av * bv, dv + p); break;
    case OP_MAX_PLUS: PANEL_LOOP(av + bv, (dv < p) ? p : dv); break;
    case OP_MAX_MIN: PANEL_LOOP((bv < av) ? bv : av, (dv < p) ? p : dv); break;
    case OP_MAX_MUL: PANEL_LOOP(av * bv, (dv < p) ? p : dv); break;
    case OP_MIN_MUL: PANEL_LOOP(av * bv, (p < dv) ? p : dv); break;
    case OP_MIN_MAX: PANEL_LOOP((av < bv) ? bv : av, (p < dv) ? p : dv); break;
    case OP_MINUS_SQUARE: PANEL_LOOP((av - bv) * (av - bv), dv + p); break;
    default: break;
  }
  if (do_epilogue) {
    for (int i = r0; i < r1; i++)
      for (int j = 0; j < N; j++) {
        size_t x = (size_t)i * N + j;
        D[x] = f_add(op, D[x], C[x]);
      }
  }
}

/* int or_and (bin_or, bin_and), kernel/host_srgemm.h:77-85 */
static void srgemm_i32_rows(int r0, int r1, int N, int K, const int32_t* A, const int32_t* B,
                            const int32_t* C, int32_t* D, int do_epilogue) {
  for (int i = r0; i < r1; i++) {
    int32_t* d = D + (size_t)i * N;
    const int32_t* a = A + (size_t)i * K;
    for (int k = 0; k < K; k++) {
      const int32_t av = a[k] != 0;
      const int32_t* b = B + (size_t)k * N;
      for (int j = 0; j < N; j++) d[j] = (d[j] != 0) || (av && (b[j] != 0));
    }
  }
  if (do_epilogue)
    for (int i = r0; i < r1; i++)
      for (int j = 0; j < N; j++) {
        size_t x = (size_t)i * N + j;
        D[x] = (D[x] != 0) || (C[x] != 0);
      }
}

/* uint8 or_and: same operators on 0/1 bytes (any nonzero byte is true). */
static void srgemm_u8_rows(int r0, int r1, int N, int K, const uint8_t* A, const uint8_t* B,
                           const uint8_t* C, uint8_t* D, int do_epilogue) {
  for (int i = r0; i < r1; i++) {
    uint8_t* d = D + (size_t)i * N;
    const uint8_t* a = A + (size_t)i * K;
    for (int k = 0; k < K; k++) {
      if (!a[k]) continue; /* bin_and(0, x) == 0 and bin_or(d, 0) == d */
      const uint8_t* b = B + (size_t)k * N;
      for (int j = 0; j < N; j++) d[j] = (uint8_t)((d[j] != 0) | (b[j] != 0));
    }
    if (K > 0) /* every k step of bin_or yields a 0/1 value */
      for (int j = 0; j < N; j++) d[j] = (uint8_t)(d[j] != 0);
  }
  if (do_epilogue)
    for (int i = r0; i < r1; i++)
      for (int j = 0; j < N; j++) {
        size_t x = (size_t)i * N + j;
        D[x] = (uint8_t)((D[x] != 0) || (C[x] != 0));
      }
}

/* FP64 error oracle for the two summing semirings (plus_mul, minus_square). */
static void srgemm_f64_rows(int op, int r0, int r1, int N, int K, const float* A, const float* B,
                            const float* C, double* D, int do_epilogue) {
  for (int i = r0; i < r1; i++) {
    double* d = D + (size_t)i * N;
    const float* a = A + (size_t)i * K;
    for (int k = 0; k < K; k++) {
      const double av = a[k];
      const float* b = B + (size_t)k * N;
      if (op == OP_MINUS_SQUARE)
        for (int j = 0; j < N; j++) { double t = av - (double)b[j]; d[j] += t * t; }
      else
        for (int j = 0; j < N; j++) d[j] += av * (double)b[j];
    }
    if (do_epilogue)
      for (int j = 0; j < N; j++) d[j] += (double)C[(size_t)i * N + j];
  }
}

/* ------------------------------------------------------------------ */
/* row-panel threading                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
  int kind; /* 0 f32, 1 i32, 2 u8, 3 f64 */
  int op, r0, r1, N, K, do_epilogue;
  const void *A, *B, *C;
  void* D;
} job_t;

static void* run_job(void* p) {
  job_t* j = (job_t*)p;
  switch (j->kind) {
    case 0: srgemm_f32_rows(j->op, j->r0, j->r1, j->N, j->K, j->A, j->B, j->C, j->D, j->do_epilogue); break;
    case 1: srgemm_i32_rows(j->r0, j->r1, j->N, j->K, j->A, j->B, j->C, j->D, j->do_epilogue); break;
    case 2: srgemm_u8_rows(j->r0, j->r1, j->N, j->K, j->A, j->B, j->C, j->D, j->do_epilogue); break;
    case 3: srgemm_f64_rows(j->op, j->r0, j->r1, j->N, j->K, j->A, j->B, j->C, j->D, j->do_epilogue); break;
  }
  return NULL;
}

static void run_panels(int kind, int op, int M, int N, int K, const void* A, const void* B, const void* C,
                       void* D, int do_epilogue, int nthreads) {
  if (M <= 0 || N <= 0) return;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > M) nthreads = M;
  if (nthreads > 256) nthreads = 256;
  job_t jobs[256];
  pthread_t th[256];
  for (int t = 0; t < nthreads; t++) {
    jobs[t] = (job_t){kind, op, (int)((int64_t)M * t / nthreads), (int)((int64_t)M * (t + 1) / nthreads),
                      N, K, do_epilogue, A, B, C, D};
  }
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, run_job, &jobs[t]);
  run_job(&jobs[0]);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
}

/* D accumulates in place, exactly as mmo::host_srgemm does: the caller
 * pre-fills D (the semiring's add-identity for a plain product). */
void oracle_srgemm_f32(int op, int M, int N, int K, const float* A, const float* B, const float* C, float* D,
                       int do_epilogue, int nthreads) {
  run_panels(0, op, M, N, K, A, B, C, D, do_epilogue, nthreads);
}
void oracle_srgemm_i32(int M, int N, int K, const int32_t* A, const int32_t* B, const int32_t* C, int32_t* D,
                       int do_epilogue, int nthreads) {
  run_panels(1, OP_OR_AND, M, N, K, A, B, C, D, do_epilogue, nthreads);
}
void oracle_srgemm_u8(int M, int N, int K, const uint8_t* A, const uint8_t* B, const uint8_t* C, uint8_t* D,
                      int do_epilogue, int nthreads) {
  run_panels(2, OP_OR_AND, M, N, K, A, B, C, D, do_epilogue, nthreads);
}
void oracle_srgemm_f64(int op, int M, int N, int K, const float* A, const float* B, const float* C, double* D,
                       int do_epilogue, int nthreads) {
  run_panels(3, op, M, N, K, A, B, C, D, do_epilogue, nthreads);
}

/* ------------------------------------------------------------------ */
/* closure by repeated squaring                                         */
/* ------------------------------------------------------------------ */
/* One closure step is Xnew = X (+) (X (x) X): the reference passes X as
 * A, B and C with do_epilogue = true and D = Xnew
 * (apps/apsp/cuASR/apsp_cuASR.cu:45-50).  The loop ends when the change
 * test reports no change or after max_iter steps; the returned count
 * includes the final, unchanged step, as the reference's num_itr does.
 *
 * tol_mode 0: bitwise unchanged.
 * tol_mode 1: reference float test, |prev-cur| > 1e-4 counts as a change
 *             (kernel/converge.cuh:9; inf-inf is NaN and counts as no change).
 * tol_mode 2: APLP variant: values in (-1,1) of the new matrix become
 *             -FLT_MAX first, then any difference counts (converge.cuh:32-43). */
int oracle_closure_f32(int op, int n, float* X, int max_iter, int tol_mode, int nthreads) {
  size_t nn = (size_t)n * n;
  float* Xn = (float*)malloc(nn * sizeof(float));
  float ident = (op == OP_MIN_PLUS || op == OP_MIN_MUL || op == OP_MIN_MAX) ? INFINITY
              : (op == OP_PLUS_MUL || op == OP_MINUS_SQUARE) ? 0.0f : -INFINITY;
  int it = 0, changed = 1;
  while (changed && it < max_iter) {
    it++;
    for (size_t x = 0; x < nn; x++) Xn[x] = ident;
    oracle_srgemm_f32(op, n, n, n, X, X, X, Xn, 1, nthreads);
    changed = 0;
    for (size_t x = 0; x < nn; x++) {
      float cur = Xn[x];
      if (tol_mode == 2 && cur > -1.0f && cur < 1.0f) cur = -3.402823466e+38f;
      if (tol_mode == 1) {
        if (fabsf(X[x] - cur) > 0.0001f) changed = 1;
      } else {
        uint32_t a, b;
        memcpy(&a, &X[x], 4);
        memcpy(&b, &cur, 4);
        if (a != b) changed = 1;
      }
      X[x] = cur;
    }
  }
  free(Xn);
  return it;
}

/* Closure with a predecessor matrix (the Floyd-Warshall baselines' pred,
 * apps/maxrp/baseline/lib/apsp.cpp:11-25, initial values main.cpp:80-94),
 * by repeated squaring: per step and (i, j), best = addop over k = 0..n-1 of
 * mulop(X[i][k], X[k][j]) with the host_srgemm accumulation, witness k* = the
 * k of the last replacement (the lowest k attaining best, as replacements
 * need a strictly better product); X'[i][j] = addop(best, X[i][j]);
 * P'[i][j] = P[k*][j] when best is strictly better than X[i][j], else
 * P[i][j].  init_pred: P[i][j] = i for i != j and X[i][j] not the add
 * identity, else -1.  Returns the step count (the final unchanged step
 * included).  Min/max-add semirings only; single-threaded. */
int oracle_closure_pred_f32(int op, int n, float* X, int32_t* P, int init_pred, int max_iter) {
  const int is_min = (op == OP_MIN_PLUS || op == OP_MIN_MUL || op == OP_MIN_MAX);
  const float ident = is_min ? INFINITY : -INFINITY;
  size_t nn = (size_t)n * n;
  if (init_pred)
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        uint32_t a, b;
        memcpy(&a, &X[(size_t)i * n + j], 4);
        memcpy(&b, &ident, 4);
        P[(size_t)i * n + j] = (i != j && a != b) ? i : -1;
      }
  float* Xn = (float*)malloc(nn * sizeof(float) + 1);
  int32_t* Pn = (int32_t*)malloc(nn * sizeof(int32_t) + 1);
  float* best = (float*)malloc((size_t)n * sizeof(float) + 1);
  int* kb = (int*)malloc((size_t)n * sizeof(int) + 1);
  int it = 0, changed = 1;
  while (changed && it < max_iter) {
    it++;
    changed = 0;
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < n; j++) {
        best[j] = ident;
        kb[j] = -1;
      }
      for (int k = 0; k < n; k++) {
        const float av = X[(size_t)i * n + k];
        const float* b = X + (size_t)k * n;
        for (int j = 0; j < n; j++) {
          const float bv = b[j];
          float p;
          switch (op) {
            case OP_MIN_PLUS: case OP_MAX_PLUS: p = av + bv; break;
            case OP_MAX_MIN: p = (bv < av) ? bv : av; break;
            case OP_MIN_MAX: p = (av < bv) ? bv : av; break;
            default: p = av * bv; break; /* max_mul, min_mul */
          }
          const int repl = is_min ? (p < best[j]) : (best[j] < p);
          if (repl) {
            best[j] = p;
            kb[j] = k;
          }
        }
      }
      for (int j = 0; j < n; j++) {
        const size_t x = (size_t)i * n + j;
        const float cv = X[x], bv = best[j];
        const float xn = is_min ? s_min(bv, cv) : s_max(bv, cv);
        const int improved = is_min ? (bv < cv) : (cv < bv);
        Xn[x] = xn;
        Pn[x] = improved ? P[(size_t)kb[j] * n + j] : P[x];
        uint32_t a, b2;
        memcpy(&a, &xn, 4);
        memcpy(&b2, &cv, 4);
        if (a != b2) changed = 1;
      }
    }
    memcpy(X, Xn, nn * sizeof(float));
    memcpy(P, Pn, nn * sizeof(int32_t));
  }
  free(Xn);
  free(Pn);
  free(best);
  free(kb);
  return it;
}

int oracle_closure_u8(int n, uint8_t* X, int max_iter, int nthreads) {
  size_t nn = (size_t)n * n;
  uint8_t* Xn = (uint8_t*)malloc(nn);
  int it = 0, changed = 1;
  while (changed && it < max_iter) {
    it++;
    memset(Xn, 0, nn);
    oracle_srgemm_u8(n, n, n, X, X, X, Xn, 1, nthreads);
    changed = memcmp(X, Xn, nn) != 0;
    memcpy(X, Xn, nn);
  }
  free(Xn);
  return it;
}

/* ------------------------------------------------------------------ */
/* k-NN: squared distances, k smallest per query, sqrt of the kept ones  */
/* ------------------------------------------------------------------ */
/* query: Q x dim row-major, ref: R x dim row-major.  Outputs are Q x k
 * row-major (query-major; the reference's layout is the transpose, k x Q).
 * Distances are accumulated in double; selection keeps the k smallest
 * with the lower reference index first among equal distances, which is
 * what the modified insertion sort produces (strict '>' shifts and the
 * '>=' skip test, apps/pld/emulation/knncuda.cu:205-216).  The returned
 * distance is sqrt of the double sum, rounded to float. */
typedef struct {
  const float *q, *r;
  int Q, R, D, k, q0, q1;
  float* out_d;
  int32_t* out_i;
  double* out_d64;
} knn_job_t;

static void* knn_run(void* p) {
  knn_job_t* j = (knn_job_t*)p;
  double* bd = (double*)malloc(sizeof(double) * (size_t)j->k);
  int32_t* bi = (int32_t*)malloc(sizeof(int32_t) * (size_t)j->k);
  for (int qi = j->q0; qi < j->q1; qi++) {
    const float* q = j->q + (size_t)qi * j->D;
    int cnt = 0;
    for (int ri = 0; ri < j->R; ri++) {
      const float* r = j->r + (size_t)ri * j->D;
      double s = 0.0;
      for (int d = 0; d < j->D; d++) { double t = (double)q[d] - (double)r[d]; s += t * t; }
      if (cnt == j->k && s >= bd[j->k - 1]) continue;
      int pos = cnt < j->k ? cnt : j->k - 1;
      while (pos > 0 && bd[pos - 1] > s) { bd[pos] = bd[pos - 1]; bi[pos] = bi[pos - 1]; pos--; }
      bd[pos] = s;
      bi[pos] = ri;
      if (cnt < j->k) cnt++;
    }
    for (int t = 0; t < j->k; t++) {
      double v = t < cnt ? bd[t] : INFINITY;
      if (j->out_d64) j->out_d64[(size_t)qi * j->k + t] = v;
      j->out_d[(size_t)qi * j->k + t] = (float)sqrt(v);
      j->out_i[(size_t)qi * j->k + t] = t < cnt ? bi[t] : -1;
    }
  }
  free(bd);
  free(bi);
  return NULL;
}

void oracle_knn(const float* query, int Q, const float* ref, int R, int dim, int k, float* out_dist,
                int32_t* out_idx, double* out_sqdist64, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > Q) nthreads = Q > 0 ? Q : 1;
  if (nthreads > 256) nthreads = 256;
  knn_job_t jobs[256];
  pthread_t th[256];
  for (int t = 0; t < nthreads; t++)
    jobs[t] = (knn_job_t){query, ref, Q, R, dim, k, (int)((int64_t)Q * t / nthreads),
                          (int)((int64_t)Q * (t + 1) / nthreads), out_dist, out_idx, out_sqdist64};
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, knn_run, &jobs[t]);
  knn_run(&jobs[0]);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
}
