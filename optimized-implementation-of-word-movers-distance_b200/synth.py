"""Seeded synthetic inputs standing in for the reference's missing data.

The reference runs on the first 100k fastText crawl-300d vectors and the
dbpedia corpus (prep.py:18-50, readme.python), neither of which is available.
These generators reproduce their shapes and value distributions:

* embeddings: C Gaussian cluster centres N(0, 0.1^2)^d, each word = a random
  centre + N(0, 0.05^2)^d, stored FP32;
* word frequencies: Zipf(s=1.1) over ranks 1..V mapped to ids 0..V-1 (the
  fastText file is frequency-sorted and prep.py keeps its head);
* source document: i.i.d. Zipf tokens until v_r distinct ids are seen,
  weights = counts / total tokens;
* target documents: per column nnz ~ U[lo, hi] distinct Zipf ids drawn without
  replacement, value 1/nnz (prep.py:38-48's set-of-tokens normalisation), ids
  ascending within a column.

Targets come back as a CSC triple (col_ptr int64[N+1], row_inds int64[nnz],
vals float64[nnz]); a source histogram as a dense float64 vector of length V.
"""
from __future__ import annotations

import dataclasses

import numpy as np

ZIPF_S = 1.1


def embeddings(V: int, d: int = 300, n_centres: int = 1000, seed: int = 0,
               chunk: int = 1 << 16) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, 0.1, size=(n_centres, d)).astype(np.float32)
    which = rng.integers(0, n_centres, size=V)
    out = np.empty((V, d), np.float32)
    for b in range(0, V, chunk):
        e = min(V, b + chunk)
        noise = rng.normal(0.0, 0.05, size=(e - b, d)).astype(np.float32)
        out[b:e] = centres[which[b:e]] + noise
    return out


def zipf_cdf(V: int, s: float = ZIPF_S) -> np.ndarray:
    p = np.arange(1, V + 1, dtype=np.float64) ** (-s)
    c = np.cumsum(p)
    return c / c[-1]


def _draw(rng, cdf, size):
    ids = np.searchsorted(cdf, rng.random(size), side="right")
    return np.minimum(ids, cdf.size - 1)


def source_doc(V: int, v_r: int, seed: int, cdf: np.ndarray | None = None
               ) -> np.ndarray:
    """Dense FP64 histogram with exactly v_r non-zeros."""
    if v_r > V:
        raise ValueError("v_r > V")
    cdf = zipf_cdf(V) if cdf is None else cdf
    rng = np.random.default_rng(seed)
    counts: dict[int, int] = {}
    total = 0
    while len(counts) < v_r:
        for t in _draw(rng, cdf, 256):
            t = int(t)
            total += 1
            counts[t] = counts.get(t, 0) + 1
            if len(counts) == v_r:
                break
    r = np.zeros(V, np.float64)
    for t, c in counts.items():
        r[t] = c / total
    return r


def targets(V: int, N: int, nnz_lo: int = 8, nnz_hi: int = 256, seed: int = 2,
            cdf: np.ndarray | None = None, chunk: int = 4096):
    """CSC target matrix, per-column nnz ~ U[nnz_lo, nnz_hi]."""
    cdf = zipf_cdf(V) if cdf is None else cdf
    rng = np.random.default_rng(seed)
    nnz = rng.integers(nnz_lo, nnz_hi + 1, size=N)
    nnz = np.minimum(nnz, V)
    col_ptr = np.zeros(N + 1, np.int64)
    col_ptr[1:] = np.cumsum(nnz)
    row_inds = np.empty(int(col_ptr[-1]), np.int64)
    for b in range(0, N, chunk):
        e = min(N, b + chunk)
        need = nnz[b:e]
        cols = _distinct_rows(rng, cdf, need)
        for k, ids in enumerate(cols):
            j = b + k
            row_inds[col_ptr[j]:col_ptr[j + 1]] = ids
    vals = np.repeat(1.0 / np.maximum(nnz, 1), nnz).astype(np.float64)
    return col_ptr, row_inds, vals


_CDF_CACHE: dict = {}


def _targets_chunk(args):
    V, lo, hi, seed, c, n = args
    cdf = _CDF_CACHE.get(V)
    if cdf is None:
        cdf = _CDF_CACHE[V] = zipf_cdf(V)
    rng = np.random.default_rng([seed, c])
    nnz = np.minimum(rng.integers(lo, hi + 1, size=n), V)
    rows = _distinct_rows(rng, cdf, nnz)
    return nnz, np.concatenate(rows) if rows else np.zeros(0, np.int64)


def targets_parallel(V: int, N: int, nnz_lo: int = 8, nnz_hi: int = 512,
                     seed: int = 2, workers: int = 0, chunk: int = 16384):
    """The same distribution as targets(), generated in chunks of `chunk`
    documents by a process pool (spawned processes; each chunk seeded by
    (seed, chunk index), so the result does not depend on the worker count;
    the Zipf(1.1) distribution over V words).  For target sets of ~1e6
    documents, where targets() takes minutes."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os
    nch = (N + chunk - 1) // chunk
    jobs = [(V, nnz_lo, nnz_hi, seed, c, min(chunk, N - c * chunk)) for c in range(nch)]
    workers = workers or max(1, min(len(jobs), (os.cpu_count() or 1)))
    with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        parts = list(ex.map(_targets_chunk, jobs))
    nnz = np.concatenate([p[0] for p in parts])
    col_ptr = np.zeros(N + 1, np.int64)
    col_ptr[1:] = np.cumsum(nnz)
    row_inds = np.concatenate([p[1] for p in parts]).astype(np.int64)
    vals = np.repeat(1.0 / np.maximum(nnz, 1), nnz).astype(np.float64)
    return col_ptr, row_inds, vals


def _distinct_rows(rng, cdf, need):
    """For each requested count, that many distinct Zipf ids in draw order
    (sequential sampling without replacement), returned sorted."""
    n = need.size
    width = int(max(need.max(), 1) * 3)
    out = [None] * n
    pending = np.arange(n)
    while pending.size:
        S = _draw(rng, cdf, (pending.size, width))
        order = np.argsort(S, axis=1, kind="stable")
        srt = np.take_along_axis(S, order, axis=1)
        first = np.ones_like(srt, dtype=bool)
        first[:, 1:] = srt[:, 1:] != srt[:, :-1]
        isfirst = np.zeros_like(first)
        np.put_along_axis(isfirst, order, first, axis=1)
        rank = np.cumsum(isfirst, axis=1)
        still = []
        for k, row in enumerate(pending):
            m = int(need[row])
            keep = isfirst[k] & (rank[k] <= m)
            ids = S[k][keep]
            if ids.size < m:
                still.append(row)
                continue
            out[row] = np.sort(ids)
        pending = np.array(still, dtype=np.int64)
        width *= 2
    return out


@dataclasses.dataclass
class Problem:
    """One source document against a target set."""
    vecs: np.ndarray      # [V, d] float32
    r: np.ndarray         # [V] float64
    col_ptr: np.ndarray   # [N+1] int64
    row_inds: np.ndarray  # [nnz] int64
    vals: np.ndarray      # [nnz] float64
    lam: float = 10.0
    max_iter: int = 15

    @property
    def V(self):
        return self.vecs.shape[0]

    @property
    def d(self):
        return self.vecs.shape[1]

    @property
    def N(self):
        return self.col_ptr.size - 1

    @property
    def nnz(self):
        return int(self.col_ptr[-1])

    @property
    def v_r(self):
        return int(np.count_nonzero(self.r))


def single_source(V=100_000, d=300, N=5000, v_r=32, nnz_lo=8, nnz_hi=256,
                  n_centres=1000, query=0, lam=10.0, max_iter=15) -> Problem:
    """The one-source plain workload: V=1e5, d=300, v_r=32, N=5000,
    nnz ~ U[8,256], lambda=10, 15 iterations (defaults)."""
    cdf = zipf_cdf(V)
    vecs = embeddings(V, d, n_centres, seed=0)
    r = source_doc(V, v_r, seed=1 + query, cdf=cdf)
    col_ptr, row_inds, vals = targets(V, N, nnz_lo, nnz_hi, seed=2, cdf=cdf)
    return Problem(vecs, r, col_ptr, row_inds, vals, lam, max_iter)


def batched_sources(V: int, n_sources: int, vr_lo: int, vr_hi: int,
                    seed: int = 7, cdf: np.ndarray | None = None):
    """n_sources dense histograms with v_r ~ U[vr_lo, vr_hi]; source q uses
    seed 1+q for its tokens.  Returns (list of r, list of v_r)."""
    cdf = zipf_cdf(V) if cdf is None else cdf
    rng = np.random.default_rng(seed)
    vrs = rng.integers(vr_lo, vr_hi + 1, size=n_sources)
    rs = [source_doc(V, int(v), seed=1 + q, cdf=cdf) for q, v in enumerate(vrs)]
    return rs, [int(v) for v in vrs]


def case(V: int, d: int, N: int, v_r: int, nnz_lo: int, nnz_hi: int,
         n_centres: int = 100, seed: int = 0, lam: float = 10.0,
         max_iter: int = 15, empty_every: int = 0) -> Problem:
    """A small seeded problem for parity tests.  Every `empty_every`-th
    document (if > 0) is left empty."""
    cdf = zipf_cdf(V)
    vecs = embeddings(V, d, n_centres, seed=seed)
    r = source_doc(V, v_r, seed=seed + 1, cdf=cdf)
    col_ptr, row_inds, vals = targets(V, N, nnz_lo, nnz_hi, seed=seed + 2,
                                      cdf=cdf)
    if empty_every > 0:
        lens = np.diff(col_ptr)
        keep = np.ones(N, bool)
        keep[::empty_every] = False
        lens = np.where(keep, lens, 0)
        mask = np.repeat(keep, np.diff(col_ptr))
        row_inds, vals = row_inds[mask], vals[mask]
        col_ptr = np.zeros(N + 1, np.int64)
        col_ptr[1:] = np.cumsum(lens)
    return Problem(vecs, r, col_ptr, row_inds, vals, lam, max_iter)


def digest(p: Problem) -> str:
    """SHA-256 of a problem's arrays (pins fixtures to the generator)."""
    import hashlib
    h = hashlib.sha256()
    for a in (p.vecs.astype(np.float32), p.r, p.col_ptr.astype(np.int64),
              p.row_inds.astype(np.int64), p.vals):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()
