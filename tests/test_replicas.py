"""Replica coordination of bench.py on two gloo ranks (CPU): every rank
reports the slowest rank's time and the whole-job throughput counts every
replica's rays."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 100.0 + 50.0 * rank
        total = bench.max_over_ranks(mine, dist, "cpu")
        out[rank] = (total, bench.job_mrays(world, 1_000_000, 10, total))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_replica():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert out[0][0] == 150.0 and out[1][0] == 150.0
    # 2 replicas x 1e6 rays x 10 steps in 150 ms.
    assert out[0][1] == pytest.approx(2 * 1e6 * 10 / 0.15 / 1e6)


def test_single_process_is_identity():
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
