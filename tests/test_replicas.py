"""Multi-rank host path on CPU (gloo, world size 2): sharding a batch by system
gives, rank by rank, exactly the solution of the whole batch (systems are
independent), and the timing reduction is the max over ranks."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from filtered_tdma_b200.replicas import local_systems, whole_job_rate


def test_local_systems_cover_batch():
    for n_sys, world, align in [(10, 2, 2), (262144, 8, 2), (1001, 3, 4), (5, 4, 2), (1, 2, 2)]:
        spans = [local_systems(n_sys, r, world, align) for r in range(world)]
        assert spans[0][0] == 0
        assert sum(c for _, c in spans) == n_sys
        for (f0, c0), (f1, _) in zip(spans, spans[1:]):
            assert f1 == f0 + c0
        for f, c in spans[:-1]:
            assert f % align == 0 and (c % align == 0 or f + c == n_sys)
    assert whole_job_rate(100, 4, 2.0) == 4 * 100 / 2e-3


def _worker(rank, world, port, results):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from filtered_tdma_b200 import workloads as W
    from filtered_tdma_b200.replicas import local_systems, max_over_ranks
    from oracle import oracle as O
    A, B, C, D = W.diag_dominant(37, 64, seed=7)
    f, c = local_systems(37, rank, world)
    sl = slice(f, f + c)
    x = O.pascal(A[:, sl], B[:, sl], C[:, sl], D[:, sl], 4)
    m = max_over_ranks(1.0 + rank)
    results[rank] = (f, c, x, m)
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_shard_by_system(orc):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        port = 29500 + os.getpid() % 1000
        mp.start_processes(_worker, args=(2, port, results), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(results)
    from filtered_tdma_b200 import workloads as W
    A, B, C, D = W.diag_dominant(37, 64, seed=7)
    whole = orc.pascal(A, B, C, D, 4)
    got = np.zeros_like(whole)
    for r in (0, 1):
        f, c, x, m = res[r]
        got[:, f:f + c] = x
        assert m == 2.0  # max over ranks of (1 + rank)
    assert np.array_equal(got, whole)
