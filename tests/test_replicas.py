"""Replicas on CPU: two gloo ranks each hash their nnz-balanced share of the
rows with the oracle; the shares put together equal the whole, and the timing
reduction takes the slowest rank."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, result_dir):
    import sys
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import oracle as O
    from minhashcuda_b200.replicas import max_over_ranks, shard_rows, sum_over_ranks
    from wmh_testlib import gamma_params, random_csr
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    rng = np.random.default_rng(123)
    dim = 400
    params = gamma_params(rng, dim, 32)
    m = random_csr(rng, 333, dim, 20, long_rows=[(5, 390)], empty_frac=0.05)
    r0, r1 = shard_rows(m.indptr, world, rank)
    part = O.COracle(*params).hash(m.data, m.indices, m.indptr[r0:r1 + 1])
    parts = [None] * world
    dist.all_gather_object(parts, (r0, r1, part))
    slowest = max_over_ranks(float(rank + 1), dist)
    total = sum_over_ranks(float(r1 - r0), dist)
    dist.barrier()
    if rank == 0:
        whole = O.COracle(*params).hash_csr(m)
        parts.sort(key=lambda p: p[0])
        assert parts[0][0] == 0 and parts[-1][1] == m.shape[0]
        for a, b in zip(parts, parts[1:]):
            assert a[1] == b[0]
        np.testing.assert_array_equal(np.concatenate([p[2] for p in parts]), whole)
        assert slowest == float(world)
        assert total == float(m.shape[0])
        open(os.path.join(result_dir, "ok"), "w").write("ok")
    dist.destroy_process_group()


def test_shard_rows_balances_nnz():
    from minhashcuda_b200.replicas import shard_rows
    ip = np.cumsum([0] + [1] * 100 + [1000] + [1] * 100)
    cuts = [shard_rows(ip, 4, r) for r in range(4)]
    assert cuts[0][0] == 0 and cuts[-1][1] == 201
    assert all(a[1] == b[0] for a, b in zip(cuts, cuts[1:]))
    assert shard_rows(ip, 1, 0) == (0, 201)
    assert shard_rows(np.array([0, 0, 0]), 3, 2)[1] == 2  # empty rows only


def test_two_gloo_ranks_reassemble_the_whole(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "ok").exists()
