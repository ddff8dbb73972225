"""The multi-GPU bookkeeping of bench.py (one process per GPU, independent
replicas, no collective on the data path) with world size 2 over gloo on the
CPU: rank discovery, the barrier, the max-over-ranks timing and the
whole-job throughput."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, REPO)
    import bench
    import torch.distributed as dist

    r, w, local = bench.setup_dist(world)
    try:
        bench.barrier(w)
        # rank r "took" 100 + 50 r ms: every rank must see the slowest
        slowest = bench.max_over_ranks(100.0 + 50.0 * r, w, "cpu")
        out[r] = (r, w, local, slowest, bench.replica_throughput(1_000_000, w, slowest))
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_and_throughput():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (rank, w, local, slowest, rate) in res.items():
        assert (rank, w, local) == (r, world, r)
        assert slowest == 150.0
        # 2 replicas x 1M queries in 150 ms (the slower rank)
        assert rate == pytest.approx(2_000_000 / 0.150 / 1e6)


def test_single_process_is_world_one():
    sys.path.insert(0, REPO)
    import bench

    if "RANK" in os.environ:
        pytest.skip("launched under a process-group launcher")
    assert bench.setup_dist(1) == (0, 1, 0)
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(500_000, 1, 250.0) == pytest.approx(2.0)
