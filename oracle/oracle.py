"""ctypes bindings for the CPU oracle (test infrastructure only).

Sign convention: every function here takes the positive regulariser
``lam`` (K = exp(-lam * M)).  ``reference_sinkhorn`` converts it to each
reference variant's own ``lamda`` argument: the fused solver computes
``exp(M * lamda)`` (sinkhorn_wmd_fused.cpp:217) and is called with ``-lam``;
the nonfused solver computes ``exp(-M * lamda)``
(sinkhorn_wmd_nonfused.cpp:172-173) and is called with ``+lam``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_U64P = ctypes.POINTER(ctypes.c_uint64)
_F64P = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int)


class OracleUnavailable(RuntimeError):
    pass


def oracle_lib_path() -> str:
    return os.path.join(_HERE, "liboracle.so")


def _ref_lib_path(variant: str) -> str:
    return os.path.join(_HERE, "_ref", f"libref_{variant}.so")


def reference_available(variant: str = "fused") -> bool:
    return os.path.exists(_ref_lib_path(variant))


_libs: dict = {}


def _load(path: str, build_target: str | None = None):
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path) and build_target is not None:
        subprocess.run(["make", "-C", _HERE, build_target], check=True,
                       stdout=subprocess.DEVNULL)
    if not os.path.exists(path):
        raise OracleUnavailable(f"{path} is not built")
    lib = ctypes.CDLL(path)
    _libs[path] = lib
    return lib


def _oracle():
    lib = _load(oracle_lib_path(), "oracle")
    if not getattr(lib, "_typed", False):
        lib.oracle_select.restype = ctypes.c_uint64
        lib.oracle_select.argtypes = [_F64P, ctypes.c_uint64, _U64P, _F64P]
        lib.oracle_sinkhorn.restype = ctypes.c_longlong
        lib.oracle_sinkhorn.argtypes = [
            _F64P, _F64P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
            _U64P, _U64P, _F64P, ctypes.c_double, ctypes.c_int, _F64P,
            ctypes.c_int]
        lib.oracle_sinkhorn_converged.restype = ctypes.c_longlong
        lib.oracle_sinkhorn_converged.argtypes = [
            _F64P, _F64P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
            _U64P, _U64P, _F64P, ctypes.c_double, ctypes.c_double,
            ctypes.c_int, _F64P, _I32P, _F64P, _F64P, ctypes.c_int]
        lib.oracle_counting_sort.restype = ctypes.c_int
        lib.oracle_counting_sort.argtypes = [
            ctypes.c_uint64, ctypes.c_uint64, _U64P, _U64P, _F64P, _U64P,
            _U64P, _F64P]
        lib.oracle_csr_to_csc.restype = ctypes.c_int
        lib.oracle_csr_to_csc.argtypes = [
            ctypes.c_uint64, ctypes.c_uint64, _U64P, _U64P, _F64P, _U64P,
            _U64P, _F64P]
        lib._typed = True
    return lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def select(r):
    """Ids with r != 0 in ascending order and their weights (fused:45-63)."""
    r = _f64(r)
    ids = np.empty(r.size + 1, np.uint64)
    w = np.empty(r.size + 1, np.float64)
    n = _oracle().oracle_select(_p(r, _F64P), r.size, _p(ids, _U64P), _p(w, _F64P))
    return ids[:n].copy(), w[:n].copy()


def sinkhorn(r, vecs, col_ptr, row_inds, vals, lam, max_iter, nthreads=0):
    """Fixed-count FP64 solve; returns WMD[N] (float64)."""
    r, vecs = _f64(r), _f64(vecs)
    col_ptr, row_inds, vals = _u64(col_ptr), _u64(row_inds), _f64(vals)
    V, d = vecs.shape
    N = col_ptr.size - 1
    out = np.empty(max(N, 1), np.float64)
    rc = _oracle().oracle_sinkhorn(
        _p(r, _F64P), _p(vecs, _F64P), V, d, N, _p(col_ptr, _U64P),
        _p(row_inds, _U64P), _p(vals, _F64P), float(lam), int(max_iter),
        _p(out, _F64P), int(nthreads))
    if rc < 0:
        raise MemoryError("oracle_sinkhorn failed")
    return out[:N]


def sinkhorn_converged(r, vecs, col_ptr, row_inds, vals, lam, tol=1e-7,
                       max_iter_cap=10000, want_u=False, nthreads=0):
    """Converged FP64 solve: returns (wmd, iters, residual, u or None)."""
    r, vecs = _f64(r), _f64(vecs)
    col_ptr, row_inds, vals = _u64(col_ptr), _u64(row_inds), _f64(vals)
    V, d = vecs.shape
    N = col_ptr.size - 1
    vr = int(np.count_nonzero(r))
    out = np.empty(max(N, 1), np.float64)
    iters = np.empty(max(N, 1), np.int32)
    res = np.empty(max(N, 1), np.float64)
    u = np.empty(max(N * vr, 1), np.float64) if want_u else None
    rc = _oracle().oracle_sinkhorn_converged(
        _p(r, _F64P), _p(vecs, _F64P), V, d, N, _p(col_ptr, _U64P),
        _p(row_inds, _U64P), _p(vals, _F64P), float(lam), float(tol),
        int(max_iter_cap), _p(out, _F64P), _p(iters, _I32P), _p(res, _F64P),
        _p(u, _F64P) if want_u else None, int(nthreads))
    if rc < 0:
        raise MemoryError("oracle_sinkhorn_converged failed")
    return (out[:N], iters[:N], res[:N],
            u[: N * vr].reshape(N, vr) if want_u else None)


def counting_sort(nkeys, key, other, w):
    """Stable counting sort of an edge list by key -> (ptr, other, w)."""
    key, other, w = _u64(key), _u64(other), _f64(w)
    nnz = key.size
    ptr = np.empty(nkeys + 1, np.uint64)
    oo = np.empty(max(nnz, 1), np.uint64)
    wo = np.empty(max(nnz, 1), np.float64)
    rc = _oracle().oracle_counting_sort(
        nkeys, nnz, _p(key, _U64P), _p(other, _U64P), _p(w, _F64P),
        _p(ptr, _U64P), _p(oo, _U64P), _p(wo, _F64P))
    if rc != 0:
        raise ValueError(f"counting sort failed ({rc})")
    return ptr, oo[:nnz], wo[:nnz]


def csc_from_csr(nrows, ncols, row_ptr, col_inds, vals):
    """Stable CSR(word-major) -> CSC(doc-major) transpose."""
    row_ptr, col_inds, vals = _u64(row_ptr), _u64(col_inds), _f64(vals)
    nnz = int(row_ptr[-1])
    col_ptr = np.empty(ncols + 1, np.uint64)
    ri = np.empty(max(nnz, 1), np.uint64)
    vo = np.empty(max(nnz, 1), np.float64)
    rc = _oracle().oracle_csr_to_csc(
        nrows, ncols, _p(row_ptr, _U64P), _p(col_inds, _U64P),
        _p(vals, _F64P), _p(col_ptr, _U64P), _p(ri, _U64P), _p(vo, _F64P))
    if rc != 0:
        raise ValueError(f"csr->csc failed ({rc})")
    return col_ptr, ri[:nnz], vo[:nnz]


def csr_from_csc(nrows, ncols, col_ptr, row_inds, vals):
    """Stable CSC(doc-major) -> CSR(word-major) transpose."""
    col_ptr, row_inds = _u64(col_ptr), _u64(row_inds)
    cols = np.repeat(np.arange(ncols, dtype=np.uint64),
                     np.diff(col_ptr).astype(np.int64))
    return counting_sort(nrows, row_inds, cols, vals)


def _ref(variant):
    lib = _load(_ref_lib_path(variant))
    if not getattr(lib, "_typed", False):
        lib.ref_sinkhorn.restype = ctypes.c_int
        lib.ref_sinkhorn.argtypes = [
            _F64P, _F64P, _F64P, ctypes.c_double, ctypes.c_int,
            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _U64P, _U64P,
            _F64P, ctypes.c_uint64, ctypes.c_int]
        lib.ref_embedding_width.restype = ctypes.c_int
        lib._typed = True
    return lib


def reference_sinkhorn(r, vecs, row_ptr, col_inds, vals, N, lam, max_iter,
                       variant="fused", nthreads=0):
    """Run the reference's own solver.  The target matrix is passed as the
    word-major CSR its globals expect (sinkhorn_wmd_fused.cpp:13) with N
    documents.  Embeddings narrower than the reference's compile-time width
    (common.h:25) are zero-padded, which leaves every distance bit-identical.
    Returns WMD[N]."""
    lib = _ref(variant)
    width = lib.ref_embedding_width()
    vecs = _f64(vecs)
    V, d = vecs.shape
    if d > width:
        raise ValueError(f"reference embedding width is {width}, got {d}")
    if d < width:
        vecs = np.ascontiguousarray(np.pad(vecs, ((0, 0), (0, width - d))))
    r = _f64(r)
    row_ptr, col_inds, vals = _u64(row_ptr), _u64(col_inds), _f64(vals)
    lamda = -float(lam) if variant == "fused" else float(lam)
    out = np.empty(int(N) + 1, np.float64)
    vr = lib.ref_sinkhorn(
        _p(r, _F64P), _p(vecs, _F64P), _p(out, _F64P), lamda, int(max_iter),
        V, int(N), width, _p(row_ptr, _U64P), _p(col_inds, _U64P),
        _p(vals, _F64P), int(row_ptr[-1]), int(nthreads))
    if vr < 0:
        raise RuntimeError(f"reference harness failed ({vr})")
    return out[: int(N)]
