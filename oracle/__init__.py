"""CPU oracle for the SIMD2 srgemm contract -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only as the checker.  The product library
(``simd2_b200`` / ``libsimd2.so``) never imports or calls it.

Two CPU implementations live here:

* ``liboracle.so`` -- ``simd2_oracle.c``, a plain-C restatement of
  ``mmo::host_srgemm`` (escalab/SIMD2 ``kernel/host_srgemm.h:17-85``), the
  closure loop (``apps/apsp/cuASR/apsp_cuASR.cu:42-54`` with
  ``kernel/converge.cuh:6-69``) and k-NN selection
  (``apps/pld/baseline/test.cpp:132-182``).
* ``_ref/libref.so`` -- the reference's own ``host_srgemm`` compiled from the
  reference header (``oracle/Makefile``); present wherever it was built.

All matrices are row-major numpy arrays.  ``srgemm`` follows host_srgemm
exactly: D accumulates in place, so a plain product starts from D filled with
the semiring's add-identity.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

OPS = ("min_plus", "plus_mul", "max_plus", "max_min", "max_mul", "min_mul", "min_max", "or_and",
       "minus_square")
OP_ID = {name: i for i, name in enumerate(OPS)}
MIN_ADD = ("min_plus", "min_mul", "min_max")
MAX_ADD = ("max_plus", "max_min", "max_mul")
SUM_ADD = ("plus_mul", "minus_square")


def add_identity(op: str) -> float:
    """The semiring's add-identity (+inf for min, -inf for max, 0 for sums/or)."""
    if op in MIN_ADD:
        return np.inf
    if op in MAX_ADD:
        return -np.inf
    return 0.0


def _load(path: str):
    return ctypes.CDLL(path) if os.path.exists(path) else None


_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and _ref/libref.so where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        P, I = ctypes.c_void_p, ctypes.c_int
        _lib.oracle_srgemm_f32.argtypes = [I, I, I, I, P, P, P, P, I, I]
        _lib.oracle_srgemm_i32.argtypes = [I, I, I, P, P, P, P, I, I]
        _lib.oracle_srgemm_u8.argtypes = [I, I, I, P, P, P, P, I, I]
        _lib.oracle_srgemm_f64.argtypes = [I, I, I, I, P, P, P, P, I, I]
        _lib.oracle_closure_f32.argtypes = [I, I, P, I, I, I]
        _lib.oracle_closure_f32.restype = I
        _lib.oracle_closure_u8.argtypes = [I, P, I, I]
        _lib.oracle_closure_u8.restype = I
        _lib.oracle_closure_pred_f32.argtypes = [I, I, P, P, I, I]
        _lib.oracle_closure_pred_f32.restype = I
        _lib.oracle_knn.argtypes = [P, I, P, I, I, I, P, P, P, I]
    return _lib


def ref_lib():
    """The reference's own host_srgemm (None where it was never built)."""
    global _ref
    if _ref is None:
        _ref = _load(os.path.join(_HERE, "_ref", "libref.so"))
        if _ref is not None:
            P, I = ctypes.c_void_p, ctypes.c_int
            _ref.ref_srgemm_f32.argtypes = [I, I, I, I, P, P, P, P, I, I]
            _ref.ref_srgemm_f32.restype = I
            _ref.ref_srgemm_i32_orand.argtypes = [I, I, I, P, P, P, P, I, I]
            _ref.ref_srgemm_i32_orand.restype = I
    return _ref


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _threads(threads):
    return threads if threads else (os.cpu_count() or 1)


def srgemm(op: str, A, B, C=None, D=None, do_epilogue=False, threads=None, use_ref=False):
    """host_srgemm semantics: returns D_in (+) A(x)B [(+) C].

    ``D`` defaults to the add-identity.  float32 for the float semirings,
    int32 or uint8 for or_and.  ``use_ref`` runs the reference's own compiled
    host_srgemm instead of the restatement.
    """
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    M, K = A.shape
    K2, N = B.shape
    assert K == K2
    if op == "or_and":
        dt = A.dtype
        assert dt in (np.int32, np.uint8)
        Dm = np.zeros((M, N), dt) if D is None else np.array(D, dtype=dt, copy=True)
        Cm = np.zeros((M, N), dt) if C is None else np.ascontiguousarray(C, dtype=dt)
        if use_ref:
            assert dt == np.int32
            ref_lib().ref_srgemm_i32_orand(M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(Dm), int(do_epilogue),
                                           _threads(threads))
        elif dt == np.int32:
            lib().oracle_srgemm_i32(M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(Dm), int(do_epilogue),
                                    _threads(threads))
        else:
            lib().oracle_srgemm_u8(M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(Dm), int(do_epilogue),
                                   _threads(threads))
        return Dm
    A = A.astype(np.float32, copy=False)
    B = B.astype(np.float32, copy=False)
    Dm = np.full((M, N), add_identity(op), np.float32) if D is None else np.array(D, np.float32, copy=True)
    Cm = np.zeros((M, N), np.float32) if C is None else np.ascontiguousarray(C, dtype=np.float32)
    if use_ref:
        rc = ref_lib().ref_srgemm_f32(OP_ID[op], M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(Dm), int(do_epilogue),
                                      _threads(threads))
        assert rc == 0
    else:
        lib().oracle_srgemm_f32(OP_ID[op], M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(Dm), int(do_epilogue),
                                _threads(threads))
    return Dm


def srgemm_f64(op: str, A, B, C=None, do_epilogue=False, threads=None):
    """FP64 error oracle for plus_mul / minus_square (float inputs, double sums)."""
    assert op in SUM_ADD
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    N = B.shape[1]
    D = np.zeros((M, N), np.float64)
    Cm = np.zeros((M, N), np.float32) if C is None else np.ascontiguousarray(C, dtype=np.float32)
    lib().oracle_srgemm_f64(OP_ID[op], M, N, K, _ptr(A), _ptr(B), _ptr(Cm), _ptr(D), int(do_epilogue),
                            _threads(threads))
    return D


def closure(op: str, X, max_iter=500, tol_mode=0, threads=None):
    """Repeated squaring X <- X (+) X(x)X until unchanged; returns (X, iterations)."""
    if op == "or_and":
        Xc = np.array(X, np.uint8, copy=True)
        it = lib().oracle_closure_u8(Xc.shape[0], _ptr(Xc), max_iter, _threads(threads))
        return Xc, it
    Xc = np.array(X, np.float32, copy=True)
    it = lib().oracle_closure_f32(OP_ID[op], Xc.shape[0], _ptr(Xc), max_iter, tol_mode, _threads(threads))
    return Xc, it


def closure_pred(op: str, X, P=None, max_iter=500):
    """Closure with a predecessor matrix: returns (X, P int32, iterations).
    P=None initialises it from X (i for an edge, -1 otherwise and on the diagonal)."""
    Xc = np.array(X, np.float32, copy=True)
    n = Xc.shape[0]
    Pc = np.zeros((n, n), np.int32) if P is None else np.array(P, np.int32, copy=True)
    it = lib().oracle_closure_pred_f32(OP_ID[op], n, _ptr(Xc), _ptr(Pc), int(P is None), max_iter)
    return Xc, Pc, it


def path(P, i, j):
    """Vertices of the recorded path i -> j from a predecessor matrix ([] when none)."""
    if i == j:
        return [i]
    out = [j]
    while j != i:
        j = int(P[i][j])
        if j < 0 or len(out) > len(P):
            return []
        out.append(j)
    return out[::-1]


def mst(W):
    """Kruskal over every edge of the undirected graph W (weight of {u, v} =
    min(W[u][v], W[v][u]), +inf = none) in (weight, u, v) order: (edges
    [m, 2] with u < v in Kruskal order, weights [m])."""
    W = np.asarray(W, np.float32)
    n = W.shape[0]
    S = np.minimum(W, W.T)
    iu, ju = np.triu_indices(n, 1)
    w = S[iu, ju]
    keep = np.isfinite(w)
    iu, ju, w = iu[keep], ju[keep], w[keep]
    order = np.lexsort((ju, iu, w))
    parent = list(range(n))

    def find(v):
        while parent[v] != v:
            parent[v] = parent[parent[v]]
            v = parent[v]
        return v

    edges, weights = [], []
    for e in order:
        a, b = find(int(iu[e])), find(int(ju[e]))
        if a != b:
            parent[b] = a
            edges.append((int(iu[e]), int(ju[e])))
            weights.append(w[e])
    return np.array(edges, np.int32).reshape(-1, 2), np.array(weights, np.float32)


def knn(query, ref, k, threads=None):
    """k nearest references per query: (dist[Q,k] float32, idx[Q,k] int32, sqdist[Q,k] float64)."""
    query = np.ascontiguousarray(query, dtype=np.float32)
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    Q, dim = query.shape
    R = ref.shape[0]
    dist = np.zeros((Q, k), np.float32)
    idx = np.zeros((Q, k), np.int32)
    sq = np.zeros((Q, k), np.float64)
    lib().oracle_knn(_ptr(query), Q, _ptr(ref), R, dim, k, _ptr(dist), _ptr(idx), _ptr(sq), _threads(threads))
    return dist, idx, sq
