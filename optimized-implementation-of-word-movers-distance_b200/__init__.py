"""B200 Sinkhorn Word Mover's Distance engine — host-side Python layer.

Everything here marshals arguments into the C ABI of libwmd_b200.so
(include/wmd_b200.h); every solve runs in the library's CUDA kernels.

Reference interfaces mirrored:

* ``sinkhorn_wmd(r, c, vecs, lamb, max_iter)`` — the Python reference
  ``main.py:37-86`` (same arguments, same ``lamb`` sign convention
  K = exp(M * lamb) of ``main.py:65``, same 1 x N matrix result).
* ``sinkhorn_wmd_fused`` / ``sinkhorn_wmd_nonfused`` — the C++ solvers
  ``sinkhorn_wmd_fused.cpp:112`` / ``sinkhorn_wmd_nonfused.cpp:114`` with their
  own ``lamda`` conventions (exp(M*lamda) and exp(-M*lamda) respectively) and
  the word-major CSR the reference keeps in its global ``c_csr``.
* ``Engine`` — the resident-corpus handle API (no reference counterpart).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import synth  # noqa: F401
from ._native import (  # noqa: F401
    CDIST_MODES, CSC, CSR, WMDError, check, exported_names, lib, LIB_PATH)

__all__ = ["sinkhorn_wmd", "sinkhorn_wmd_fused", "sinkhorn_wmd_nonfused",
           "sinkhorn_wmd_csc", "Engine", "WMDError", "synth"]


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _csc_struct(V, N, col_ptr, row_inds, vals):
    keep = (col_ptr, row_inds, vals)
    s = CSC(V, N, int(col_ptr[-1]), _ptr(col_ptr, ctypes.c_uint64),
            _ptr(row_inds, ctypes.c_uint64), _ptr(vals, ctypes.c_double))
    return s, keep


def _csr_struct(V, N, row_ptr, col_inds, vals):
    keep = (row_ptr, col_inds, vals)
    s = CSR(V, N, int(row_ptr[-1]), _ptr(row_ptr, ctypes.c_uint64),
            _ptr(col_inds, ctypes.c_uint64), _ptr(vals, ctypes.c_double))
    return s, keep


def sinkhorn_wmd_csc(r, vecs, col_ptr, row_inds, vals, lamda, max_iter,
                     variant="fused"):
    """Drop-in solve with a document-major (CSC) target matrix.  ``lamda``
    follows the chosen reference variant's sign convention."""
    r, vecs = _f64(r), _f64(vecs)
    col_ptr, row_inds, vals = _u64(col_ptr), _u64(row_inds), _f64(vals)
    V, d = vecs.shape
    N = col_ptr.size - 1
    out = np.empty(N, np.float64)
    s, _keep = _csc_struct(V, N, col_ptr, row_inds, vals)
    fn = (lib().wmd_sinkhorn_fused_csc if variant == "fused"
          else lib().wmd_sinkhorn_nonfused_csc)
    check(fn(_ptr(r, ctypes.c_double), _ptr(vecs, ctypes.c_double),
             _ptr(out, ctypes.c_double), float(lamda), int(max_iter), V, N, d,
             ctypes.byref(s)))
    return out


def dropin_h2d_bytes() -> int:
    """Host -> device bytes of this thread's last drop-in call: with the
    embeddings in pinned host memory only the rows of words that occur in the
    targets or the source cross the bus (``wmd_dropin_h2d_bytes``)."""
    return int(lib().wmd_dropin_h2d_bytes())


def _csr_call(fn, r, vecs, lamda, max_iter, row_ptr, col_inds, vals, num_docs):
    r, vecs = _f64(r), _f64(vecs)
    row_ptr, col_inds, vals = _u64(row_ptr), _u64(col_inds), _f64(vals)
    V, d = vecs.shape
    out = np.empty(int(num_docs), np.float64)
    s, _keep = _csr_struct(V, int(num_docs), row_ptr, col_inds, vals)
    check(fn(_ptr(r, ctypes.c_double), _ptr(vecs, ctypes.c_double),
             _ptr(out, ctypes.c_double), float(lamda), int(max_iter), V,
             int(num_docs), d, ctypes.byref(s)))
    return out


def sinkhorn_wmd_fused(r, vecs, lamda, max_iter, row_ptr, col_inds, vals,
                       num_docs):
    """Mirror of sinkhorn_wmd (sinkhorn_wmd_fused.cpp:112): K = exp(lamda*M),
    target matrix as the reference's word-major CSR."""
    return _csr_call(lib().wmd_sinkhorn_fused, r, vecs, lamda, max_iter,
                     row_ptr, col_inds, vals, num_docs)


def sinkhorn_wmd_nonfused(r, vecs, lamda, max_iter, row_ptr, col_inds, vals,
                          num_docs):
    """Mirror of sinkhorn_wmd (sinkhorn_wmd_nonfused.cpp:114):
    K = exp(-lamda*M)."""
    return _csr_call(lib().wmd_sinkhorn_nonfused, r, vecs, lamda, max_iter,
                     row_ptr, col_inds, vals, num_docs)


def sinkhorn_wmd(r, c, vecs, lamb, max_iter):
    """Drop-in for main.py:37 ``sinkhorn_wmd(r, c, vecs, lamb, max_iter)``.

    r: dense query histogram (V,), c: scipy sparse V x N target matrix,
    vecs: V x d embeddings, lamb: K = exp(M * lamb) (main.py:65; the
    reference's default is -1).  Returns a 1 x N ``np.matrix`` as main.py's
    ``(u * ((KM) @ v)).sum(axis=0)`` does.  main.py selects r > 0
    (main.py:49); negative weights are rejected here, as the reference's C++
    driver rejects them (sinkhorn_wmd_fused.cpp:570-574).
    """
    from scipy import sparse
    c = sparse.csc_matrix(c)
    c.sort_indices()
    r = np.asarray(r, dtype=np.float64).reshape(-1)
    out = sinkhorn_wmd_csc(r, np.asarray(vecs), c.indptr, c.indices, c.data,
                           lamb, max_iter, "fused")
    return np.asmatrix(out.reshape(1, -1))


def _pack_sources(sources):
    """(ptr, ids, weights) of a list of dense histograms or (ids, weights)
    pairs, ids ascending within each source."""
    ptr = [0]
    ids, ws = [], []
    for src in sources:
        if isinstance(src, tuple):
            i, w = np.asarray(src[0], np.uint64), np.asarray(src[1], np.float64)
            order = np.argsort(i, kind="stable")
            i, w = i[order], w[order]
        else:
            r = np.asarray(src, np.float64)
            i = np.nonzero(r)[0].astype(np.uint64)
            w = r[i.astype(np.int64)]
        ids.append(i)
        ws.append(w)
        ptr.append(ptr[-1] + i.size)
    ptr = np.asarray(ptr, np.uint64)
    ids = np.ascontiguousarray(np.concatenate(ids) if ids else np.zeros(0), np.uint64)
    ws = np.ascontiguousarray(np.concatenate(ws) if ws else np.zeros(0), np.float64)
    return ptr, ids, ws


def ws_param_count(d: int) -> int:
    """Length of the warm-start parameter vector for embedding width d."""
    return int(lib().wmd_ws_param_count(int(d)))


def ws_init_params(d: int, seed: int = 0) -> np.ndarray:
    p = np.empty(ws_param_count(d), np.float32)
    check(lib().wmd_ws_init_params(int(d), int(seed), _ptr(p, ctypes.c_float)))
    return p


def read_mtx(path):
    """The reference's mat.mtx: (V, N, words, docs, weights), 0-based ids in
    file order."""
    V, N, Z = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    b = str(path).encode()
    check(lib().wmd_mtx_header(b, ctypes.byref(V), ctypes.byref(N), ctypes.byref(Z)))
    words = np.empty(Z.value, np.uint64)
    docs = np.empty(Z.value, np.uint64)
    w = np.empty(Z.value, np.float64)
    n = ctypes.c_uint64()
    check(lib().wmd_read_mtx(b, Z.value, _ptr(words, ctypes.c_uint64),
                             _ptr(docs, ctypes.c_uint64), _ptr(w, ctypes.c_double),
                             ctypes.byref(n)))
    return V.value, N.value, words, docs, w


def read_vecs(path, V: int, d: int) -> np.ndarray:
    """The reference's vecs.out: (V, d) float64."""
    out = np.empty((V, d), np.float64)
    check(lib().wmd_read_vecs(str(path).encode(), V, d, _ptr(out, ctypes.c_double)))
    return out


def read_r(path, V: int) -> np.ndarray:
    """The reference's r.out: V non-negative values."""
    out = np.empty(V, np.float64)
    check(lib().wmd_read_r(str(path).encode(), V, _ptr(out, ctypes.c_double)))
    return out


class Engine:
    """Resident-corpus solver (handle API of include/wmd_b200.h).  ``lam`` is
    the positive regulariser: K = exp(-lam * M)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        check(lib().wmd_create(ctypes.byref(self._h), int(device)))
        self.V = self.d = self.N = 0

    def close(self):
        if self._h:
            lib().wmd_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return int(lib().wmd_stream(self._h) or 0)

    @property
    def launch_count(self) -> int:
        return int(lib().wmd_last_launch_count(self._h))

    def set_embeddings(self, vecs):
        """vecs: numpy float64/float32 (V, d), or a CUDA tensor (torch) of
        either dtype on this handle's device."""
        if hasattr(vecs, "data_ptr") and getattr(vecs, "is_cuda", False):
            V, d = vecs.shape
            ptr = ctypes.c_void_p(vecs.contiguous().data_ptr())
            f = (lib().wmd_set_embeddings_f64 if str(vecs.dtype) == "torch.float64"
                 else lib().wmd_set_embeddings_f32)
            check(f(self._h, ptr, V, d, 1))
        else:
            a = np.asarray(vecs)
            if a.dtype == np.float32:
                a = np.ascontiguousarray(a)
                check(lib().wmd_set_embeddings_f32(
                    self._h, a.ctypes.data_as(ctypes.c_void_p), a.shape[0],
                    a.shape[1], 0))
            else:
                a = _f64(a)
                check(lib().wmd_set_embeddings_f64(
                    self._h, a.ctypes.data_as(ctypes.c_void_p), a.shape[0],
                    a.shape[1], 0))
            V, d = a.shape
        self.V, self.d = int(V), int(d)

    def set_embeddings_bf16(self, vecs):
        """vecs: BF16 embeddings, a torch bfloat16 tensor (CPU or this
        handle's device) or a numpy uint16 array of raw BF16 bit patterns."""
        if hasattr(vecs, "data_ptr"):
            t = vecs.contiguous()
            V, d = t.shape
            where = 1 if getattr(t, "is_cuda", False) else 0
            check(lib().wmd_set_embeddings_bf16(self._h, ctypes.c_void_p(t.data_ptr()),
                                                V, d, where))
        else:
            a = np.ascontiguousarray(vecs, np.uint16)
            V, d = a.shape
            check(lib().wmd_set_embeddings_bf16(self._h, a.ctypes.data_as(ctypes.c_void_p),
                                                V, d, 0))
        self.V, self.d = int(V), int(d)

    def set_targets(self, col_ptr, row_inds, vals, V=None):
        col_ptr, row_inds, vals = _u64(col_ptr), _u64(row_inds), _f64(vals)
        V = self.V if V is None else int(V)
        N = col_ptr.size - 1
        s, _keep = _csc_struct(V, N, col_ptr, row_inds, vals)
        check(lib().wmd_set_targets_csc(self._h, ctypes.byref(s)))
        self.N = N

    def set_targets_csr(self, row_ptr, col_inds, vals, N):
        row_ptr, col_inds, vals = _u64(row_ptr), _u64(col_inds), _f64(vals)
        V = row_ptr.size - 1
        s, _keep = _csr_struct(V, int(N), row_ptr, col_inds, vals)
        check(lib().wmd_set_targets_csr(self._h, ctypes.byref(s)))
        self.N = int(N)

    def edges_to_csc(self, words, docs, w, V: int, N: int):
        """GPU CSC build of an edge list: (col_ptr, rows, vals)."""
        words, docs, w = _u64(words), _u64(docs), _f64(w)
        cp = np.empty(N + 1, np.uint64)
        rows = np.empty(words.size, np.uint64)
        vals = np.empty(words.size, np.float64)
        check(lib().wmd_edges_to_csc(
            self._h, _ptr(words, ctypes.c_uint64), _ptr(docs, ctypes.c_uint64),
            _ptr(w, ctypes.c_double), words.size, int(V), int(N),
            _ptr(cp, ctypes.c_uint64), _ptr(rows, ctypes.c_uint64),
            _ptr(vals, ctypes.c_double)))
        return cp, rows, vals

    def set_targets_edges(self, words, docs, w, V: int, N: int):
        """Target set from an edge list (e.g. read_mtx), CSC built on the GPU."""
        words, docs, w = _u64(words), _u64(docs), _f64(w)
        check(lib().wmd_set_targets_edges(
            self._h, _ptr(words, ctypes.c_uint64), _ptr(docs, ctypes.c_uint64),
            _ptr(w, ctypes.c_double), words.size, int(V), int(N)))
        self.N = int(N)

    def set_cdist_mode(self, mode: str):
        """Cost panel: "fp32" (CUDA cores, the default), "tf32x3" (tcgen05
        tensor cores on the FP32 embeddings split into TF32 high + low
        parts: FP32-accurate), "f16x3" (tcgen05 on a resident split-FP16
        copy: FP32-accurate, single-source queries; batches use the tf32x3
        form), "fp16" / "bf16" (16-bit operands)."""
        check(lib().wmd_set_cdist_mode(self._h, CDIST_MODES[mode]))

    def set_relaxation(self, omega: float = 1.0):
        """Over-relaxation of both Sinkhorn half-steps, 0 < omega < 2, with a
        per-document guard; applies with a tolerance set (set_tolerance),
        1 = the reference's iteration."""
        check(lib().wmd_set_relaxation(self._h, float(omega)))

    def set_autotune(self, enable: bool = True):
        check(lib().wmd_set_autotune(self._h, int(bool(enable))))

    def set_block_shape(self, shape: int):
        """Pin the block solve's shape (0-2 CUDA-core launch shapes, 3-5 the
        tensor-core form at 1, 2, 4 CTAs per SM, -1 build-time default,
        -2 autotune)."""
        check(lib().wmd_set_block_shape(self._h, int(shape)))

    def autotune_choices(self) -> dict:
        """{(panel width, beyond 64 MiB): chosen block-solve launch shape}."""
        a = (ctypes.c_int * 8)()
        check(lib().wmd_autotune_choices(self._h, a))
        out = {}
        for i, v in enumerate(a):
            if v != -2:
                out[(128 * (i // 2 + 1), bool(i % 2))] = lib().wmd_block_shape_name(v).decode()
        return out

    def set_solve_precision(self, prec: str):
        """'fp32' (default) or 'bf16': K panel storage read by the iterations
        for sources with 64 < v_r <= 512."""
        check(lib().wmd_set_solve_precision(self._h, {"fp32": 0, "bf16": 1}[prec]))

    def set_batch_mode(self, stacked: bool = True, group_budget_gib: float = 32.0):
        """Batched queries in stacked groups (a fixed number of launches per
        group of same-width sources, one persistent solve over all their
        (source, document) pairs) or source by source."""
        check(lib().wmd_set_batch_mode(self._h, int(bool(stacked)),
                                       int(group_budget_gib * (1 << 30))))

    def solve_shape_choices(self) -> dict:
        """{largest v_r of the lane layout: the warp solve's tuned shape}."""
        a = (ctypes.c_int * 6)()
        check(lib().wmd_solve_shape_choices(self._h, a))
        return {32 << i: lib().wmd_solve_shape_name(v).decode()
                for i, v in enumerate(a) if v != -2}

    def group_shape_choices(self) -> dict:
        """Launch shapes of the stacked batch solves: {("block", panel width)
        or ("warp", largest v_r of the lane layout): shape name}."""
        a = (ctypes.c_int * 10)()
        check(lib().wmd_group_shape_choices(self._h, a))
        out = {}
        for i in range(4):
            if a[i] != -2:
                out[("block", 128 * (i + 1))] = lib().wmd_block_shape_name(a[i]).decode()
        for i in range(6):
            if a[4 + i] != -2:
                out[("warp", 32 << i)] = lib().wmd_solve_shape_name(a[4 + i]).decode()
        return out

    @property
    def last_batch_groups(self) -> int:
        return int(lib().wmd_last_batch_groups(self._h))

    def set_solve_order(self, order: str):
        """'document' (default: a document's scalings on chip for every pass)
        or 'word' (the reference's word-major traversal: each K row read once
        per pass, u gathered and x scattered per entry; fixed update count,
        cold start, single-source queries)."""
        check(lib().wmd_set_solve_order(self._h, {"document": 0, "word": 1}[order]))

    def query(self, r, lam: float, max_iter: int) -> np.ndarray:
        r = _f64(r)
        out = np.empty(self.N, np.float64)
        check(lib().wmd_query_dense(self._h, _ptr(r, ctypes.c_double),
                                    float(lam), int(max_iter),
                                    _ptr(out, ctypes.c_double)))
        return out

    def query_topk(self, r, lam: float, max_iter: int, k: int):
        """k nearest documents: (indices, scores), ascending WMD, ties by
        index, NaN last (numpy.argsort(scores, kind='stable')[:k])."""
        r = _f64(r)
        idx = np.empty(k, np.uint32)
        val = np.empty(k, np.float64)
        check(lib().wmd_query_topk(
            self._h, _ptr(r, ctypes.c_double), float(lam), int(max_iter), int(k),
            idx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            _ptr(val, ctypes.c_double)))
        return idx, val

    def topk_device(self, scores_dev_ptr: int, n: int, k: int, idx_dev_ptr: int,
                    val_dev_ptr: int):
        check(lib().wmd_topk_device(self._h, ctypes.c_void_p(scores_dev_ptr), n,
                                    int(k), ctypes.c_void_p(idx_dev_ptr),
                                    ctypes.c_void_p(val_dev_ptr)))

    def query_batch(self, sources, lam: float, max_iter: int,
                    want_iters: bool = False):
        """sources: list of dense histograms r (length V) or of (ids,
        weights) pairs.  Returns a (len(sources), N) array of scores (and the
        per-document iteration counts if want_iters)."""
        ptr, ids, ws = _pack_sources(sources)
        S = len(sources)
        out = np.empty((S, self.N), np.float64)
        it = np.empty((S, self.N), np.int32) if want_iters else None
        check(lib().wmd_query_batch(
            self._h, _ptr(ptr, ctypes.c_uint64), _ptr(ids, ctypes.c_uint64),
            _ptr(ws, ctypes.c_double), S, float(lam), int(max_iter),
            _ptr(out, ctypes.c_double),
            it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if want_iters else None))
        return (out, it) if want_iters else out

    # -- learned warm start -------------------------------------------------
    def ws_build_training_set(self, sources, lam: float, docs_per_source: int,
                              words_per_doc: int = 16, label_tol: float = 1e-7,
                              label_max_iter: int = 5000, seed: int = 0) -> dict:
        """Converged-FP64 labels for (source, document) pairs of the resident
        target set; returns {'rows', 'groups', 'mean_label_iters'}."""
        ptr, ids, ws = _pack_sources(sources)
        rows, groups = ctypes.c_uint64(), ctypes.c_uint64()
        mit = ctypes.c_double()
        check(lib().wmd_ws_build_training_set(
            self._h, _ptr(ptr, ctypes.c_uint64), _ptr(ids, ctypes.c_uint64),
            _ptr(ws, ctypes.c_double), len(sources), float(lam), int(docs_per_source),
            int(words_per_doc), float(label_tol), int(label_max_iter), int(seed),
            ctypes.byref(rows), ctypes.byref(groups), ctypes.byref(mit)))
        return {"rows": rows.value, "groups": groups.value,
                "mean_label_iters": mit.value}

    def ws_train(self, params, epochs: int, batch_groups: int = 256,
                 lr: float = 1e-3, seed: int = 0):
        """Adam on the built training set; returns (params, per-epoch loss)."""
        p = np.ascontiguousarray(params, np.float32).copy()
        loss = np.empty(int(epochs), np.float64)
        check(lib().wmd_ws_train(self._h, _ptr(p, ctypes.c_float), int(epochs),
                                 int(batch_groups), float(lr), int(seed),
                                 _ptr(loss, ctypes.c_double)))
        return p, loss

    def ws_loss_grad(self, d: int, X, t, gptr, params):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        gptr = np.ascontiguousarray(gptr, np.int64)
        params = np.ascontiguousarray(params, np.float32)
        grad = np.empty_like(params)
        loss = ctypes.c_double()
        check(lib().wmd_ws_loss_grad(
            self._h, int(d), _ptr(X, ctypes.c_float), _ptr(t, ctypes.c_float),
            gptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), gptr.size - 1,
            _ptr(params, ctypes.c_float), ctypes.byref(loss), _ptr(grad, ctypes.c_float)))
        return loss.value, grad

    def ws_training_set(self, info: dict) -> dict:
        """The built training set (from ws_build_training_set's info):
        standardised X, labels y, group pointers, per-group source index and
        document, per-row source-word index."""
        rows, groups = int(info["rows"]), int(info["groups"])
        d = int(self.d)
        F = ((2 * d + 5) + 15) // 16 * 16
        X = np.empty((rows, F), np.float32)
        y = np.empty(rows, np.float32)
        gptr = np.empty(groups + 1, np.int64)
        gs = np.empty(groups, np.uint32)
        gd = np.empty(groups, np.uint32)
        rw = np.empty(rows, np.int32)
        u32 = ctypes.POINTER(ctypes.c_uint32)
        check(lib().wmd_ws_get_training_set(
            self._h, _ptr(X, ctypes.c_float), _ptr(y, ctypes.c_float),
            gptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            gs.ctypes.data_as(u32), gd.ctypes.data_as(u32),
            rw.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return {"X": X, "y": y, "gptr": gptr, "source": gs, "doc": gd, "word": rw}

    def set_warm_start(self, params):
        """Start queries from the model's prediction (None: cold start)."""
        if params is None:
            check(lib().wmd_set_warm_start(self._h, None))
        else:
            p = np.ascontiguousarray(params, np.float32)
            check(lib().wmd_set_warm_start(self._h, _ptr(p, ctypes.c_float)))

    def ws_init_scalings(self, r, lam: float) -> np.ndarray:
        """The model's initial scalings u0 [N][v_r] for a dense source r."""
        r = _f64(r)
        vr_max = int(np.count_nonzero(r))
        u0 = np.empty((self.N, max(vr_max, 1)), np.float32)
        vr = ctypes.c_uint64()
        check(lib().wmd_ws_init_scalings(self._h, _ptr(r, ctypes.c_double), float(lam),
                                         _ptr(u0, ctypes.c_float), ctypes.byref(vr)))
        return u0[:, :vr.value]

    def query_device(self, r_dev_ptr: int, vr_cap: int, lam: float,
                     max_iter: int, out_dev_ptr: int):
        """Asynchronous solve on device pointers (e.g. torch ``data_ptr()``)
        on the handle's stream; call ``check()`` to synchronise."""
        check(lib().wmd_query_dense_device(
            self._h, ctypes.c_void_p(r_dev_ptr), int(vr_cap), float(lam),
            int(max_iter), ctypes.c_void_p(out_dev_ptr)))

    def check(self):
        check(lib().wmd_check(self._h))

    def selftest_bounded_wait(self, limit_ns: int) -> int:
        """Run the bounded-wait self-test (a device wait that can only end
        through its limit) and return the status the next check reports
        (WMD_ERR_DEVICE_TIMEOUT = 7 when the wait gave up as designed)."""
        check(lib().wmd_selftest_bounded_wait(self._h, int(limit_ns)))
        return int(lib().wmd_check(self._h))

    def set_tolerance(self, tol: float):
        """0: fixed max_iter updates (the reference); > 0: stop each document
        once its marginal residual is <= tol (max_iter becomes a cap)."""
        check(lib().wmd_set_tolerance(self._h, float(tol)))

    def last_iterations(self) -> np.ndarray:
        it = np.empty(self.N, np.int32)
        check(lib().wmd_last_iterations(
            self._h, it.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return it

    def set_timing(self, enable: bool = True):
        check(lib().wmd_set_timing(self._h, int(bool(enable))))

    def stage_times(self):
        """(select_ms, cdist_ms, solve_ms) of the last query (synchronises)."""
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(lib().wmd_stage_times(self._h, ctypes.byref(a), ctypes.byref(b),
                                    ctypes.byref(c)))
        return a.value, b.value, c.value
