"""simd2_b200 -- B200-native semiring GEMM (srgemm) engine.

Host-side Python mirror of the escalab/SIMD2 srgemm operator surface.  Every
call goes through the C ABI of ``libsimd2.so`` (``include/simd2.h``), which
launches hand-written sm_100a kernels; there is no CPU or PyTorch fallback.
If the library is missing or the device is not sm_100, calls raise.

Tensors are torch CUDA tensors (plumbing only: device memory and streams).
Row-major semantics follow ``mmo::host_srgemm`` (kernel/host_srgemm.h:17-49):
``D = id (+) A(x)B`` and, with ``do_epilogue``, ``D = D (+) C``.
"""
from __future__ import annotations

import ctypes
import os

import torch

from .build import LIB as _LIB_PATH

OPS = ("min_plus", "plus_mul", "max_plus", "max_min", "max_mul", "min_mul", "min_max", "or_and",
       "minus_square")
OP_ID = {name: i for i, name in enumerate(OPS)}
CONV = {"exact": 0, "tol": 1, "aplp": 2}

STATUS = {
    0: "ok", 1: "invalid argument", 2: "unsupported operation", 3: "CUDA runtime error",
    4: "workspace allocation failed", 5: "device-side wait timed out",
    6: "closure did not converge within max_iter", 7: "no sm_100 device",
    8: "scratch or capacity limit exceeded",
}


class Simd2Error(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: simd2 status {status} ({STATUS.get(status, 'unknown')})")


class NotConverged(Simd2Error):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Load libsimd2.so (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"libsimd2.so not built at {_LIB_PATH}; run `python -m simd2_b200.build`")
        L = ctypes.CDLL(_LIB_PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        L.simd2_srgemm.argtypes = [I, I, I, I, P, I, P, I, P, I, P, I, I, P]
        L.simd2_srgemm_orand_i32.argtypes = [I, I, I, P, I, P, I, P, I, P, I, I, P]
        L.simd2_srgemm_orand_u8.argtypes = [I, I, I, P, I, P, I, P, I, P, I, I, P]
        L.simd2_closure.argtypes = [I, I, P, I, I, I, ctypes.POINTER(I), P]
        L.simd2_closure_orand_u8.argtypes = [I, P, I, I, ctypes.POINTER(I), P]
        L.simd2_closure_panel_step.argtypes = [I, I, I, P, I, P, I, P, I, I, P, P]
        L.simd2_closure_pred.argtypes = [I, I, P, I, P, I, I, I, ctypes.POINTER(I), P]
        LL = ctypes.c_longlong
        L.simd2_spgemm_nnz.argtypes = [I, I, I, I, P, P, I, P, P, I, P, P, I, P, ctypes.POINTER(LL), P]
        L.simd2_spgemm_compute.argtypes = [I, I, I, I, P, P, P, I, P, P, P, I, P, P, P, I, P, P, P, LL, P]
        L.simd2_closure_sparse.argtypes = [I, I, P, P, P, LL, ctypes.POINTER(LL), I, ctypes.POINTER(I), P]
        L.simd2_mst.argtypes = [I, P, I, P, P, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(I), P]
        L.simd2_reserve_workspace.argtypes = [I, I, I, I, P, ctypes.POINTER(ctypes.c_size_t)]
        L.simd2_release_workspaces.argtypes = []
        L.simd2_device_status.argtypes = []
        L.simd2_status_string.argtypes = [I]
        L.simd2_status_string.restype = ctypes.c_char_p
        L.simd2_version.restype = ctypes.c_char_p
        PI = ctypes.POINTER(I)
        PF = ctypes.POINTER(ctypes.c_float)
        L.simd2_srgemm_tuned.argtypes = [I, I, I, I, P, I, P, I, P, I, P, I, I, I, P]
        L.simd2_closure_ex.argtypes = [I, I, P, I, I, I, I, I, P, PI, PI, PF, PF, P]
        L.simd2_mlp_param_count.argtypes = []
        L.simd2_mlp_forward.argtypes = [P, P, I, P, P]
        L.simd2_mlp_gradient.argtypes = [P, P, P, I, P, P, P]
        L.simd2_mlp_adam.argtypes = [P, P, P, P, ctypes.c_float, I, P]
        L.simd2_batched_plan_create.argtypes = [I, I, ctypes.POINTER(P), PI, PI, I, I, ctypes.POINTER(P)]
        L.simd2_batched_plan_run.argtypes = [P, P]
        L.simd2_batched_plan_iters.argtypes = [P, PI, PI]
        L.simd2_batched_plan_destroy.argtypes = [P]
        L.simd2_closure_batched.argtypes = [I, I, ctypes.POINTER(P), PI, PI, I, I, PI, P]
        L.simd2_srgemm_f16.argtypes = [I, I, I, I, P, I, P, I, P, I, P, I, I, P]
        L.simd2_set_dense_configs.argtypes = [ctypes.POINTER(I), ctypes.POINTER(I), I]
        L.simd2_knn.argtypes = [P, I, I, P, I, I, I, I, P, P, I, P]
        L.simd2_knn.restype = I
        L.simd2_knn_ex.argtypes = [P, I, I, P, I, I, I, I, P, P, I, I, P]
        L.simd2_knn_ex.restype = I
        L.simd2_selftest_timeout.argtypes = [ctypes.c_uint]
        L.simd2_selftest_timeout.restype = I
        L.simd2_timeout_site.argtypes = []
        L.simd2_timeout_site.restype = I
        L.simd2_launch_count.argtypes = []
        L.simd2_launch_count.restype = ctypes.c_longlong
        L.simd2_profile_begin.argtypes = []
        L.simd2_profile_result.argtypes = [I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.simd2_profile_result.restype = I
        L.simd2_profile_end.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_longlong)]
        for name in ("simd2_srgemm", "simd2_srgemm_orand_i32", "simd2_srgemm_orand_u8", "simd2_closure",
                     "simd2_closure_orand_u8", "simd2_reserve_workspace", "simd2_release_workspaces",
                     "simd2_device_status", "simd2_profile_begin", "simd2_profile_end",
                     "simd2_batched_plan_create", "simd2_batched_plan_run", "simd2_batched_plan_iters",
                     "simd2_batched_plan_destroy", "simd2_closure_batched", "simd2_srgemm_tuned",
                     "simd2_closure_ex", "simd2_mlp_param_count", "simd2_mlp_forward", "simd2_mlp_gradient",
                     "simd2_mlp_adam", "simd2_srgemm_f16", "simd2_set_dense_configs"):
            getattr(L, name).restype = I
        _lib = L
    return _lib


def _stream(stream) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _check(rc: int, what: str):
    if rc == 6:
        raise NotConverged(rc, what)
    if rc != 0:
        raise Simd2Error(rc, what)


def _mat(t: torch.Tensor, name: str) -> int:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dim() != 2:
        raise ValueError(f"{name} must be 2-D")
    if t.numel() == 0:
        return max(t.size(1), 1)
    if t.stride(1) != 1 and t.size(1) > 1:
        raise ValueError(f"{name} must be a 2-D row-major tensor with unit column stride")
    return t.stride(0) if t.size(0) > 1 else max(t.size(1), 1)


def srgemm(op: str, A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, do_epilogue: bool = False,
           D: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """D = id (+) A(x)B [(+) C] on the GPU; returns D (allocated if not given).

    float32 tensors for the eight float semirings; int32 or uint8 for or_and.
    """
    M, K = A.shape
    K2, N = B.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    if D is None:
        D = torch.empty((M, N), dtype=A.dtype, device=A.device)
    lda, ldb, ldd = _mat(A, "A"), _mat(B, "B"), _mat(D, "D")
    if do_epilogue:
        if C is None:
            raise ValueError("do_epilogue needs C")
        ldc = _mat(C, "C")
        cptr = C.data_ptr()
    else:
        ldc, cptr = N, None
    s = _stream(stream)
    if op == "or_and":
        fn = {torch.int32: lib().simd2_srgemm_orand_i32, torch.uint8: lib().simd2_srgemm_orand_u8}.get(A.dtype)
        if fn is None:
            raise TypeError("or_and takes int32 or uint8 tensors")
        rc = fn(M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb, cptr, ldc, D.data_ptr(), ldd, int(do_epilogue), s)
    else:
        for t, nm in ((A, "A"), (B, "B"), (D, "D")):
            if t.dtype != torch.float32:
                raise TypeError(f"{nm} must be float32 for {op}")
        rc = lib().simd2_srgemm(OP_ID[op], M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb, cptr, ldc, D.data_ptr(),
                                ldd, int(do_epilogue), s)
    _check(rc, f"srgemm({op})")
    return D


def srgemm_f16(op: str, A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, do_epilogue: bool = False,
               D: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """srgemm with float16 A and B and float32 C / D: the entry behind the
    reference's ``tensor_srgemm`` (kernel/tensor_srgemm.cuh:197-218).  The
    halves are widened exactly; or_and reads any nonzero as true and writes 0/1."""
    M, K = A.shape
    K2, N = B.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    if A.dtype != torch.float16 or B.dtype != torch.float16:
        raise TypeError("srgemm_f16 takes float16 A and B")
    if D is None:
        D = torch.empty((M, N), dtype=torch.float32, device=A.device)
    if D.dtype != torch.float32 or (do_epilogue and (C is None or C.dtype != torch.float32)):
        raise TypeError("srgemm_f16 takes float32 C and D")
    cptr, ldc = (C.data_ptr(), _mat(C, "C")) if do_epilogue else (None, N)
    rc = lib().simd2_srgemm_f16(OP_ID[op], M, N, K, A.data_ptr(), _mat(A, "A"), B.data_ptr(), _mat(B, "B"), cptr, ldc,
                                D.data_ptr(), _mat(D, "D"), int(do_epilogue), _stream(stream))
    _check(rc, f"srgemm_f16({op})")
    return D


NUM_CONFIGS = 8
DISPATCH = {"dense": 0, "fixed": 1, "learned": 2, "rules": 3}
SPARSE_CONFIG = NUM_CONFIGS  # a CSR SpGEMM closure step


def config_id(split: int, skip: bool) -> int:
    """Kernel configuration of the CUDA-core path: split-K factor and block skipping."""
    return {1: 0, 2: 1, 4: 2, 8: 3}[split] | (4 if skip else 0)


def config_desc(cfg: int) -> str:
    """Name of a closure-step configuration; NUM_CONFIGS marks a sparse (SpGEMM) step of the learned policy."""
    if cfg == NUM_CONFIGS:
        return "sparse"
    return f"split{1 << (cfg & 3)}{'+skip' if cfg >> 2 else ''}"


def srgemm_tuned(op: str, A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, do_epilogue: bool = False,
                 D: torch.Tensor | None = None, config: int = 0, stream=None) -> torch.Tensor:
    """srgemm for the min/max semirings with an explicit kernel configuration (same bits for every config)."""
    M, K = A.shape
    N = B.shape[1]
    if D is None:
        D = torch.empty((M, N), dtype=torch.float32, device=A.device)
    cptr, ldc = (C.data_ptr(), _mat(C, "C")) if do_epilogue else (None, N)
    rc = lib().simd2_srgemm_tuned(OP_ID[op], M, N, K, A.data_ptr(), _mat(A, "A"), B.data_ptr(), _mat(B, "B"), cptr,
                                  ldc, D.data_ptr(), _mat(D, "D"), int(do_epilogue), int(config), _stream(stream))
    _check(rc, f"srgemm_tuned({op}, {config})")
    return D


def set_dense_configs(table) -> None:
    """Install the plain dense path's split-K factor by size: ``table`` is a
    list of (n_min, config) with n_min ascending and config 0..3 (split
    1 << config), as ``autotune.dense_table`` measures it; [] restores the
    rule.  Every split gives the same bits."""
    table = sorted((int(n), int(c)) for n, c in table)
    ns = (ctypes.c_int * max(len(table), 1))(*[n for n, _ in table])
    cs = (ctypes.c_int * max(len(table), 1))(*[c for _, c in table])
    _check(lib().simd2_set_dense_configs(ns, cs, len(table)), "set_dense_configs")


def closure_ex(op: str, X: torch.Tensor, dispatch: str = "dense", config: int = 0, mlp_params=None,
               max_iter: int = 500, conv: str = "exact", record: bool = False, stream=None):
    """Closure with a per-step dispatch policy.

    ``dispatch``: "dense" (the plain path), "fixed" (``config`` every step;
    ``SPARSE_CONFIG`` runs CSR SpGEMM steps while X fits the sparse store,
    then the plain path), "learned" (above n = 1024, bitwise change test: the
    MLP in ``mlp_params`` chooses each step between the dense configurations
    and, while X is sparse, a CSR SpGEMM step) or "rules" (the hand-written
    policy: sparse steps under fixed entry and product thresholds, then
    ``config`` for the dense steps).  Every policy gives the same bits and
    step count.

    Returns the step count, or with ``record`` a dict with the per-step
    configurations (``SPARSE_CONFIG`` for a sparse step), device times (ms)
    and cost-model features (9 per step).
    """
    n = X.shape[0]
    it = ctypes.c_int(0)
    cfgs = (ctypes.c_int * max(max_iter, 1))()
    ms = (ctypes.c_float * max(max_iter, 1))()
    nf = 9
    feats = (ctypes.c_float * (max(max_iter, 1) * nf))()
    pp = None if mlp_params is None else ctypes.c_void_p(mlp_params.data_ptr())
    rc = lib().simd2_closure_ex(OP_ID[op], n, X.data_ptr(), _mat(X, "X"), max_iter, CONV[conv], DISPATCH[dispatch],
                                int(config), pp, ctypes.byref(it), cfgs if record else None,
                                ms if record else None, feats if record else None, _stream(stream))
    _check(rc, f"closure_ex({op}, {dispatch})")
    if not record:
        return it.value
    k = it.value
    return {"iters": k, "configs": list(cfgs)[:k], "ms": list(ms)[:k],
            "features": [list(feats)[nf * i:nf * i + nf] for i in range(k)]}


def closure(op: str, X: torch.Tensor, max_iter: int = 500, conv: str = "exact", stream=None,
            raise_not_converged: bool = True) -> int:
    """Repeated squaring X <- X (+) X(x)X in place until unchanged; returns the step count.

    or_and takes a uint8 0/1 matrix; from n = 8192 its sparse first steps run
    as CSR SpGEMM steps (same result and step count as the dense loop)."""
    n = X.shape[0]
    if X.shape != (n, n):
        raise ValueError("closure needs a square matrix")
    ldx = _mat(X, "X")
    it = ctypes.c_int(0)
    s = _stream(stream)
    if op == "or_and":
        if X.dtype != torch.uint8:
            raise TypeError("or_and closure takes a uint8 tensor")
        rc = lib().simd2_closure_orand_u8(n, X.data_ptr(), ldx, max_iter, ctypes.byref(it), s)
    else:
        if X.dtype != torch.float32:
            raise TypeError("closure takes a float32 tensor")
        rc = lib().simd2_closure(OP_ID[op], n, X.data_ptr(), ldx, max_iter, CONV[conv], ctypes.byref(it), s)
    if rc == 6 and not raise_not_converged:
        return it.value
    _check(rc, f"closure({op})")
    return it.value


def closure_pred(op: str, X: torch.Tensor, P: torch.Tensor | None = None, max_iter: int = 500, stream=None):
    """Closure of X in place with a predecessor matrix: returns (steps, P).

    P[i][j] is the vertex before j on the best i -> j path (-1: none, and on
    the diagonal).  P=None starts from the edges of X (i where X[i][j] is not
    the add identity); a given int32 P is taken as the starting state and
    updated in place.  Semirings with a min or max add."""
    n = X.shape[0]
    if X.shape != (n, n) or X.dtype != torch.float32:
        raise ValueError("closure_pred needs a square float32 matrix")
    init = P is None
    if init:
        P = torch.empty((n, n), dtype=torch.int32, device=X.device)
    elif P.shape != (n, n) or P.dtype != torch.int32:
        raise ValueError("P must be an n x n int32 tensor")
    it = ctypes.c_int(0)
    rc = lib().simd2_closure_pred(OP_ID[op], n, X.data_ptr(), _mat(X, "X"), P.data_ptr(), _mat(P, "P"), int(init),
                                  max_iter, ctypes.byref(it), _stream(stream))
    _check(rc, f"closure_pred({op})")
    return it.value, P


def path(P, i: int, j: int):
    """Vertices of the recorded i -> j path from a predecessor matrix (host
    array or tensor); [] when there is none."""
    if i == j:
        return [i]
    Ph = P.cpu().numpy() if isinstance(P, torch.Tensor) else P
    out = [j]
    while j != i:
        j = int(Ph[i][j])
        if j < 0 or len(out) > len(Ph):
            return []
        out.append(j)
    return out[::-1]


SPARSE_IDENTITY = {"min_plus": float("inf"), "max_plus": float("-inf"), "max_min": float("-inf"),
                   "min_max": float("inf"), "plus_mul": 0.0}


def csr_from_dense(X: torch.Tensor, op: str):
    """(rowptr, cols, vals) of the entries of X that are not the add identity of ``op``."""
    mask = X != SPARSE_IDENTITY[op]
    counts = mask.sum(1, dtype=torch.int32)
    rowptr = torch.zeros(X.shape[0] + 1, dtype=torch.int32, device=X.device)
    rowptr[1:] = torch.cumsum(counts, 0, dtype=torch.int32)
    cols = mask.nonzero()[:, 1].to(torch.int32).contiguous()
    return rowptr, cols, X[mask].to(torch.float32).contiguous()


def csr_to_dense(csr, n_cols: int, op: str) -> torch.Tensor:
    """Dense matrix with the add identity of ``op`` where ``csr`` stores nothing."""
    rowptr, cols, vals = csr
    rows = rowptr.numel() - 1
    X = torch.full((rows, n_cols), SPARSE_IDENTITY[op], dtype=torch.float32, device=vals.device)
    r = torch.repeat_interleave(torch.arange(rows, device=vals.device), (rowptr[1:] - rowptr[:-1]).long())
    X[r, cols.long()] = vals
    return X


def _csr(t, name):
    rowptr, cols, vals = t
    for x, dt in ((rowptr, torch.int32), (cols, torch.int32), (vals, torch.float32)):
        if x.dtype != dt or not x.is_cuda or not x.is_contiguous():
            raise TypeError(f"{name}: CSR needs contiguous CUDA int32 rowptr / cols and float32 vals")
    if cols.numel() != vals.numel():
        raise ValueError(f"{name}: cols and vals differ in length")
    return rowptr, cols, vals


def spgemm(op: str, A, B, n_cols: int, C=None, stream=None):
    """D = A (x) B [(+) C] on CSR matrices (rowptr, cols, vals); returns D as CSR.

    ``n_cols`` is the column count of B (and C, D).  Absent entries are the add
    identity (``SPARSE_IDENTITY``); columns come out sorted; values equal the
    dense srgemm's bit for bit."""
    ap, aj, av = _csr(A, "A")
    bp, bj, bv = _csr(B, "B")
    cp = cj = cv = None
    if C is not None:
        cp, cj, cv = _csr(C, "C")
    M, K = ap.numel() - 1, bp.numel() - 1
    dp = torch.empty(M + 1, dtype=torch.int32, device=av.device)
    nnz = ctypes.c_longlong(0)
    s = _stream(stream)
    ptr = lambda t: t.data_ptr() if t is not None else None
    rc = lib().simd2_spgemm_nnz(OP_ID[op], M, n_cols, K, ap.data_ptr(), aj.data_ptr(), aj.numel(), bp.data_ptr(),
                                bj.data_ptr(), bj.numel(), ptr(cp), ptr(cj), cj.numel() if cj is not None else 0,
                                dp.data_ptr(), ctypes.byref(nnz), s)
    _check(rc, f"spgemm_nnz({op})")
    dj = torch.empty(nnz.value, dtype=torch.int32, device=av.device)
    dv = torch.empty(nnz.value, dtype=torch.float32, device=av.device)
    rc = lib().simd2_spgemm_compute(OP_ID[op], M, n_cols, K, ap.data_ptr(), aj.data_ptr(), av.data_ptr(), aj.numel(),
                                    bp.data_ptr(), bj.data_ptr(), bv.data_ptr(), bj.numel(), ptr(cp), ptr(cj), ptr(cv),
                                    cj.numel() if cj is not None else 0, dp.data_ptr(), ptr(dj), ptr(dv), nnz.value, s)
    _check(rc, f"spgemm_compute({op})")
    return dp, dj, dv


def closure_sparse(op: str, X, capacity: int | None = None, max_iter: int = 500, stream=None):
    """Closure of a square CSR matrix (rowptr, cols, vals): returns (closed CSR, steps).

    ``capacity`` bounds the stored entries (default n * n); the arrays are
    copied into buffers of that size, closed in place and trimmed."""
    rowptr, cols, vals = _csr(X, "X")
    n = rowptr.numel() - 1
    cap = n * n if capacity is None else int(capacity)
    nnz0 = cols.numel()
    if cap < nnz0:
        raise ValueError("capacity below the matrix's entry count")
    rp = rowptr.clone()
    cj = torch.empty(max(cap, 1), dtype=torch.int32, device=vals.device)
    cv = torch.empty(max(cap, 1), dtype=torch.float32, device=vals.device)
    cj[:nnz0] = cols
    cv[:nnz0] = vals
    nnz = ctypes.c_longlong(nnz0)
    it = ctypes.c_int(0)
    rc = lib().simd2_closure_sparse(OP_ID[op], n, rp.data_ptr(), cj.data_ptr(), cv.data_ptr(), cap,
                                    ctypes.byref(nnz), max_iter, ctypes.byref(it), _stream(stream))
    _check(rc, f"closure_sparse({op}) [entries {nnz.value}]")
    return (rp, cj[: nnz.value].clone(), cv[: nnz.value].clone()), it.value


def mst(W: torch.Tensor, stream=None):
    """Minimum spanning forest of the undirected graph W (+inf = no edge, the
    weight of {u, v} is min(W[u][v], W[v][u])): returns (edges [m, 2] int32
    numpy with u < v, weights [m] float32 numpy, total weight, closure steps)."""
    import numpy as np
    n = W.shape[0]
    if W.shape != (n, n) or W.dtype != torch.float32:
        raise ValueError("mst needs a square float32 matrix")
    edges = np.zeros((max(n - 1, 1), 2), np.int32)
    weights = np.zeros(max(n - 1, 1), np.float32)
    cnt, it = ctypes.c_int(0), ctypes.c_int(0)
    tot = ctypes.c_double(0)
    rc = lib().simd2_mst(n, W.data_ptr() if n else None, _mat(W, "W") if n else 1,
                         edges.ctypes.data_as(ctypes.c_void_p), weights.ctypes.data_as(ctypes.c_void_p),
                         ctypes.byref(cnt), ctypes.byref(tot), ctypes.byref(it), _stream(stream))
    _check(rc, "mst")
    return edges[: cnt.value].copy(), weights[: cnt.value].copy(), tot.value, it.value


def closure_panel_step(op: str, panel: torch.Tensor, full: torch.Tensor, out: torch.Tensor, changed: torch.Tensor,
                       conv: str = "exact", stream=None) -> None:
    """out = panel (+) panel (x) full for a row panel of a distributed closure.

    ``panel`` (rows x n) holds this rank's rows of X, ``full`` (>= n rows x n)
    all rows; ``changed`` is a device int32 tensor of one element that
    becomes nonzero when ``out`` differs from ``panel``.  Asynchronous."""
    rows, n = panel.shape
    if full.shape[1] != n or full.shape[0] < n or out.shape != panel.shape:
        raise ValueError("panel step: panel rows x n, full >= n x n, out like panel")
    want = torch.uint8 if op == "or_and" else torch.float32
    if panel.dtype != want or full.dtype != want or out.dtype != want:
        raise TypeError(f"{op} panel step takes {want} tensors")
    if changed.dtype != torch.int32 or changed.numel() < 1 or changed.device != panel.device:
        raise TypeError("changed must be an int32 tensor on the panel's device")
    rc = lib().simd2_closure_panel_step(OP_ID[op], rows, n, panel.data_ptr(), _mat(panel, "panel"), full.data_ptr(),
                                        _mat(full, "full"), out.data_ptr(), _mat(out, "out"), CONV[conv],
                                        changed.data_ptr(), _stream(stream))
    _check(rc, f"closure_panel_step({op})")


class BatchedClosure:
    """Plan for closing many independent square matrices in one persistent launch.

    ``mats`` are float32 CUDA tensors (n x n, row-major) closed in place by
    ``run``.  ``run`` only launches kernels on the stream (no allocation, no
    host synchronisation), so it can be captured in a CUDA graph.
    """

    def __init__(self, op: str, mats, max_iter: int = 500, conv: str = "exact"):
        self.mats = list(mats)
        count = len(self.mats)
        ptrs = (ctypes.c_void_p * max(count, 1))(*[m.data_ptr() for m in self.mats])
        ns = (ctypes.c_int * max(count, 1))(*[m.shape[0] for m in self.mats])
        lds = (ctypes.c_int * max(count, 1))(*[_mat(m, "X") for m in self.mats])
        for m in self.mats:
            if m.dtype != torch.float32 or m.shape[0] != m.shape[1]:
                raise ValueError("batched closure takes square float32 matrices")
        self.count = count
        self._plan = ctypes.c_void_p()
        _check(lib().simd2_batched_plan_create(OP_ID[op], count, ptrs, ns, lds, max_iter, CONV[conv],
                                               ctypes.byref(self._plan)), "batched_plan_create")

    def run(self, stream=None):
        _check(lib().simd2_batched_plan_run(self._plan, _stream(stream)), "batched_plan_run")

    def iters(self):
        it = (ctypes.c_int * max(self.count, 1))()
        nc = ctypes.c_int(0)
        _check(lib().simd2_batched_plan_iters(self._plan, it, ctypes.byref(nc)), "batched_plan_iters")
        return list(it)[: self.count], nc.value

    def close(self):
        if self._plan:
            lib().simd2_batched_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def closure_batched(op: str, mats, max_iter: int = 500, conv: str = "exact", stream=None):
    """Closes every matrix of ``mats`` in place in one persistent launch; returns the step counts."""
    mats = list(mats)
    count = len(mats)
    ptrs = (ctypes.c_void_p * max(count, 1))(*[m.data_ptr() for m in mats])
    ns = (ctypes.c_int * max(count, 1))(*[m.shape[0] for m in mats])
    lds = (ctypes.c_int * max(count, 1))(*[_mat(m, "X") for m in mats])
    it = (ctypes.c_int * max(count, 1))()
    rc = lib().simd2_closure_batched(OP_ID[op], count, ptrs, ns, lds, max_iter, CONV[conv], it, _stream(stream))
    _check(rc, f"closure_batched({op})")
    return list(it)[:count]


KNN_MODES = {"auto": 0, "fused": 1, "materialised": 2}


def knn(query: torch.Tensor, ref: torch.Tensor, k: int, stream=None, mode: str = "auto"):
    """k nearest references of every query (Euclidean): (dist [Q,k] float32, idx [Q,k] int32).

    Mirrors the PLD path of the reference (minus_square srgemm, insertion-sort
    top-k, sqrt); outputs are query-major.  ``mode``: "fused" selects inside
    the distance kernel (D <= 128), "materialised" writes distance blocks and
    selects from them, "auto" picks fused when it applies; results are
    bit-identical.
    """
    Q, D = query.shape
    R, D2 = ref.shape
    if D != D2:
        raise ValueError("query and ref dimensions differ")
    if mode not in KNN_MODES:
        raise ValueError(f"unknown k-NN mode {mode!r}")
    dist = torch.empty((Q, k), dtype=torch.float32, device=query.device)
    idx = torch.empty((Q, k), dtype=torch.int32, device=query.device)
    rc = lib().simd2_knn_ex(query.data_ptr(), Q, _mat(query, "query"), ref.data_ptr(), R, _mat(ref, "ref"), D, k,
                            dist.data_ptr(), idx.data_ptr(), k, KNN_MODES[mode], _stream(stream))
    _check(rc, "knn")
    return dist, idx


def device_status() -> int:
    """Read and clear the device-side error word (0 = no kernel reported an error)."""
    return lib().simd2_device_status()


def launch_count() -> int:
    """Kernels launched by libsimd2 so far in this process."""
    return int(lib().simd2_launch_count())


class KernelTimer:
    """Times every main srgemm kernel launched inside the ``with`` block with
    CUDA events recorded on the kernel's own stream."""

    def __enter__(self):
        _check(lib().simd2_profile_begin(), "profile_begin")
        return self

    def __exit__(self, *exc):
        ms, n, ops = ctypes.c_double(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
        _check(lib().simd2_profile_end(ctypes.byref(ms), ctypes.byref(n), ctypes.byref(ops)), "profile_end")
        self.kernel_ms, self.launches, self.ops = ms.value, n.value, ops.value
        self.by_kind = {}
        for kind, name in ((0, "simt"), (1, "tensor")):
            _check(lib().simd2_profile_result(kind, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(ops)),
                   "profile_result")
            self.by_kind[name] = (ms.value, n.value, ops.value)
        return False


def version() -> str:
    return lib().simd2_version().decode()
