"""Document sharding across GPUs (one process per GPU).

A target document's WMD depends only on its own column and the shared source
panel (sinkhorn_wmd_fused.cpp:255-289 per entry, :382-393 per column), so the
target set splits into contiguous document ranges with no exchange inside
the solve.  The ranges are balanced by non-zeros, the same idea as the
reference's nnz-balanced thread chunks (sinkhorn_wmd_fused.cpp:88-109 binary
search over the row pointers, :161-193), applied to GPUs.  The only
collective is the final gather of WMD[N] (8 bytes per document).
"""
from __future__ import annotations

import numpy as np


def partition(col_ptr, parts: int):
    """Contiguous document ranges [(j0, j1), ...] with about nnz / parts
    non-zeros each (boundaries by binary search on col_ptr)."""
    col_ptr = np.asarray(col_ptr, np.int64)
    N = col_ptr.size - 1
    nnz = int(col_ptr[-1])
    bounds = [0]
    for p in range(1, parts):
        target = (nnz * p) // parts
        j = int(np.searchsorted(col_ptr, target, side="left"))
        bounds.append(min(max(j, bounds[-1]), N))
    bounds.append(N)
    return [(bounds[p], bounds[p + 1]) for p in range(parts)]


def partition_sources(vrs, parts: int):
    """Batched queries: contiguous source ranges [(s0, s1), ...] with about
    equal sum of v_r each.  A source's solve costs nnz * v_r (every target
    document against every source word), the target set being the same for
    all, so v_r is the weight; the split is the prefix-sum search of
    partition() applied to sources."""
    w = np.asarray(vrs, np.int64)
    S = w.size
    cum = np.concatenate([[0], np.cumsum(w)])
    total = int(cum[-1])
    bounds = [0]
    for p in range(1, parts):
        target = (total * p) // parts
        s = int(np.searchsorted(cum, target, side="left"))
        bounds.append(min(max(s, bounds[-1]), S))
    bounds.append(S)
    return [(bounds[p], bounds[p + 1]) for p in range(parts)]


def shard_targets(col_ptr, row_inds, vals, j0: int, j1: int):
    """CSC arrays of documents [j0, j1) (column pointers rebased to 0)."""
    col_ptr = np.asarray(col_ptr, np.int64)
    a, b = int(col_ptr[j0]), int(col_ptr[j1])
    return (col_ptr[j0:j1 + 1] - a, np.asarray(row_inds)[a:b], np.asarray(vals)[a:b])


def gather(local, group=None, device=None):
    """All ranks' shard results concatenated in rank order (every rank gets
    the full vector).  Shards may differ in length: each is padded to the
    longest before the all-gather and trimmed after."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.ascontiguousarray(local, np.float64))
    if device is not None:
        t = t.to(device)
    world = dist.get_world_size(group)
    n = torch.tensor([t.numel()], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    pad = torch.zeros(m, dtype=t.dtype, device=t.device)
    pad[: t.numel()] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return np.concatenate([p[:s].cpu().numpy() for p, s in zip(parts, sizes)])


def gather_rows(local, n_cols: int, group=None, device=None):
    """All ranks' [rows, n_cols] result blocks stacked in rank order."""
    flat = gather(np.asarray(local, np.float64).reshape(-1), group, device)
    return flat.reshape(-1, n_cols)


class ShardedSources:
    """One rank's share of a batch of source documents: the embeddings and
    the whole target set are replicated, the sources [s0, s1) of a
    v_r-balanced partition are solved on this rank's GPU, and `query_batch`
    returns every source's scores (local batch + gather)."""

    def __init__(self, vecs, col_ptr, row_inds, vals, rank: int, world: int,
                 device: int = 0):
        from . import Engine
        self.rank, self.world, self.device = rank, world, device
        self.N = len(col_ptr) - 1
        self.eng = Engine(device)
        self.eng.set_embeddings(vecs)
        self.eng.set_targets(col_ptr, row_inds, vals)

    def query_batch(self, sources, lam: float, max_iter: int, group=None):
        import torch
        vrs = [int(np.count_nonzero(r)) if np.ndim(r) == 1 else len(r[0])
               for r in sources]
        s0, s1 = partition_sources(vrs, self.world)[self.rank]
        local = (self.eng.query_batch(list(sources[s0:s1]), lam, max_iter)
                 if s1 > s0 else np.zeros((0, self.N)))
        return gather_rows(local, self.N, group, torch.device("cuda", self.device))

    def close(self):
        self.eng.close()


class ShardedEngine:
    """One rank's share of a target set: the embeddings are replicated, the
    documents [j0, j1) of an nnz-balanced partition are resident on this
    rank's GPU, and `query` returns the full WMD vector (local solve +
    gather)."""

    def __init__(self, vecs, col_ptr, row_inds, vals, rank: int, world: int,
                 device: int = 0):
        from . import Engine
        self.rank, self.world = rank, world
        self.j0, self.j1 = partition(col_ptr, world)[rank]
        self.eng = Engine(device)
        self.eng.set_embeddings(vecs)
        cp, ri, vv = shard_targets(col_ptr, row_inds, vals, self.j0, self.j1)
        self.local_n = self.j1 - self.j0
        self.has_nnz = self.local_n > 0 and cp[-1] > 0
        if self.has_nnz:
            self.eng.set_targets(cp, ri, vv)
        self.device = device

    def query_local(self, r, lam: float, max_iter: int):
        if self.local_n == 0:
            return np.zeros(0)
        if not self.has_nnz:
            # only empty documents: NaN as in the reference (u = 1/0 times
            # x = 0, fused:382-393), 0 for an empty source
            return np.full(self.local_n, np.nan if np.count_nonzero(r) else 0.0)
        return self.eng.query(r, lam, max_iter)

    def query(self, r, lam: float, max_iter: int, group=None):
        import torch
        local = self.query_local(r, lam, max_iter)
        return gather(local, group, torch.device("cuda", self.device))

    def close(self):
        self.eng.close()
