"""CPU, world size 2 over gloo: the document-shard partition and the final
gather of the multi-GPU path.  Each rank solves its own shard with the FP64
oracle (standing in for its GPU), the gathered vector must equal the
single-process result bit for bit (documents are independent)."""
import os
import socket

import numpy as np
import pytest

PKG = "optimized-implementation-of-word-movers-distance_b200"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_balances_nnz_and_covers_all_documents():
    import importlib
    shard = importlib.import_module(PKG + ".shard")
    rng = np.random.default_rng(0)
    lens = rng.integers(0, 300, 1001)
    lens[::50] = 0
    cp = np.concatenate([[0], np.cumsum(lens)])
    for parts in (1, 2, 3, 7, 8):
        rngs = shard.partition(cp, parts)
        assert rngs[0][0] == 0 and rngs[-1][1] == 1001
        assert all(a[1] == b[0] for a, b in zip(rngs, rngs[1:]))
        loads = [cp[b] - cp[a] for a, b in rngs]
        assert max(loads) - min(loads) <= 2 * lens.max()
    # more parts than documents: empty shards, still a cover
    rngs = shard.partition(cp[:4], 8)
    assert rngs[-1][1] == 3 and sum(b - a for a, b in rngs) == 3


def test_source_partition_balances_vr():
    import importlib
    shard = importlib.import_module(PKG + ".shard")
    rng = np.random.default_rng(1)
    vrs = rng.integers(4, 513, 512)
    for parts in (1, 2, 4, 8):
        rngs = shard.partition_sources(vrs, parts)
        assert rngs[0][0] == 0 and rngs[-1][1] == 512
        assert all(a[1] == b[0] for a, b in zip(rngs, rngs[1:]))
        loads = [int(vrs[a:b].sum()) for a, b in rngs]
        assert max(loads) - min(loads) <= 2 * vrs.max()
    assert shard.partition_sources([5, 7], 4)[-1][1] == 2


def _src_worker(rank, world, port, out_path):
    import importlib
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        import sys
        repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, repo)
        import oracle
        synth = importlib.import_module(PKG + ".synth")
        shard = importlib.import_module(PKG + ".shard")
        p = synth.case(1200, 300, 60, 24, 8, 80, 40, 15)
        srcs = [synth.source_doc(p.V, v, seed=300 + q) for q, v in
                enumerate((5, 40, 12, 90, 33))]
        vrs = [int(np.count_nonzero(r)) for r in srcs]
        s0, s1 = shard.partition_sources(vrs, world)[rank]
        E = p.vecs.astype(np.float64)
        local = np.array([oracle.sinkhorn(r, E, p.col_ptr, p.row_inds, p.vals, p.lam,
                                          p.max_iter, nthreads=1) for r in srcs[s0:s1]]
                         ).reshape(-1, p.N)
        full = shard.gather_rows(local, p.N)
        if rank == 0:
            ref = np.array([oracle.sinkhorn(r, E, p.col_ptr, p.row_inds, p.vals, p.lam,
                                            p.max_iter, nthreads=1) for r in srcs])
            np.save(out_path, np.stack([full, ref]))
    finally:
        dist.destroy_process_group()


def test_gather_of_source_shards_world2(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "src.npy")
    mp.start_processes(_src_worker, args=(2, _free_port(), out), nprocs=2,
                       join=True, start_method="spawn")
    full, ref = np.load(out)
    assert full.shape == ref.shape == (5, 60)
    np.testing.assert_array_equal(full, ref)


def _worker(rank, world, port, out_path):
    import importlib
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        import sys
        repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, repo)
        import oracle
        synth = importlib.import_module(PKG + ".synth")
        shard = importlib.import_module(PKG + ".shard")
        p = synth.case(1500, 300, 201, 24, 8, 120, 40, 13, empty_every=17)
        j0, j1 = shard.partition(p.col_ptr, world)[rank]
        cp, ri, vv = shard.shard_targets(p.col_ptr, p.row_inds, p.vals, j0, j1)
        local = oracle.sinkhorn(p.r, p.vecs.astype(np.float64), cp, ri, vv, p.lam,
                                p.max_iter, nthreads=1)
        full = shard.gather(local)
        if rank == 0:
            ref = oracle.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                                  p.row_inds, p.vals, p.lam, p.max_iter, nthreads=1)
            np.save(out_path, np.stack([full, ref]))
        # uneven shards: rank 1 contributes nothing
        odd = shard.gather(np.arange(5.0) if rank == 0 else np.zeros(0))
        assert np.array_equal(odd, np.arange(5.0))
    finally:
        dist.destroy_process_group()


def test_gather_of_document_shards_world2(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2,
                       join=True, start_method="spawn")
    full, ref = np.load(out)
    assert full.shape == ref.shape
    np.testing.assert_array_equal(np.isnan(full), np.isnan(ref))
    np.testing.assert_array_equal(full[~np.isnan(full)], ref[~np.isnan(ref)])


@pytest.mark.gpu
def test_sharded_engine_single_rank_nccl(wmd, synth, oracle_mod):
    """The GPU side of the shard path at world size 1 (NCCL): the sharded
    engine's gathered result equals the plain engine's."""
    import importlib
    import torch
    import torch.distributed as dist
    shard = importlib.import_module(PKG + ".shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        p = synth.case(2000, 300, 300, 32, 8, 100, 40, 17)
        se = shard.ShardedEngine(p.vecs, p.col_ptr, p.row_inds, p.vals, 0, 1, 0)
        got = se.query(p.r, p.lam, p.max_iter)
        eng = wmd.Engine()
        eng.set_embeddings(p.vecs)
        eng.set_targets(p.col_ptr, p.row_inds, p.vals)
        np.testing.assert_array_equal(got, eng.query(p.r, p.lam, p.max_iter))
        eng.close()
        se.close()
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_sources_single_rank_nccl(wmd, synth):
    """The source-partition path at world size 1 (NCCL): the gathered batch
    equals the plain engine's batch."""
    import importlib
    import torch
    import torch.distributed as dist
    shard = importlib.import_module(PKG + ".shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        p = synth.case(2000, 300, 200, 32, 8, 100, 40, 19)
        srcs = [synth.source_doc(p.V, v, seed=500 + v) for v in (8, 70, 150)]
        ss = shard.ShardedSources(p.vecs, p.col_ptr, p.row_inds, p.vals, 0, 1, 0)
        got = ss.query_batch(srcs, p.lam, p.max_iter)
        eng = wmd.Engine()
        eng.set_embeddings(p.vecs)
        eng.set_targets(p.col_ptr, p.row_inds, p.vals)
        np.testing.assert_array_equal(got, eng.query_batch(srcs, p.lam, p.max_iter))
        eng.close()
        ss.close()
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
