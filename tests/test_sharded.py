"""Start sharding over ranks (the multi-GPU path), exercised on CPU with two
gloo ranks: shares cover the starts exactly once, the exchange picks the first
maximum in global start order and every rank ends with the same loadings."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _sharded():
    return importlib.import_module("24am_b200.sharded")


@pytest.mark.parametrize("total,world", [(10, 2), (1, 2), (1024, 8), (7, 3), (64, 1)])
def test_shards_partition_the_starts(total, world):
    sh = _sharded()
    seen = []
    for r in range(world):
        first, count = sh.shard(total, world, r)
        seen.extend(range(first, first + count))
    assert seen == list(range(total))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, fvals, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = _sharded()
        n, total = 6, 5
        starts = np.arange(n * total, dtype=np.float32).reshape(n, total, order="F")

        def solve_share(V):
            # stand-in for this rank's GPU solve: the fixed objective of the
            # test case, loadings that name the rank and its first start
            first, _ = sh.shard(total, world, rank)
            return np.full(n, 100 * rank + first, np.float32) + V[:, 0] * 0, fvals[rank]

        x, best, r, share = sh.solve_sharded(solve_share, total, starts)
        out[rank] = (x.tolist(), best, r, share)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fvals,expect_rank", [((3.0, 5.0), 1), ((5.0, 5.0), 0),
                                               ((float("nan"), 2.0), 1)])
def test_best_of_two_gloo_ranks(fvals, expect_rank):
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), fvals, out), nprocs=world,
                           join=True, start_method="spawn")
        res = dict(out)
    sh = _sharded()
    first = sh.shard(5, world, expect_rank)[0]
    for rank in range(world):
        x, best, r, share = res[rank]
        assert r == expect_rank
        assert best == fvals[expect_rank]
        assert x == [100.0 * expect_rank + first] * 6
        assert share == sh.shard(5, world, rank)
