"""The multi-GPU path of bench.py on CPU ranks (gloo, world size 2): every rank serves its
own streams (no data-path collective), and the reported time is the maximum over ranks,
so every rank derives the same whole-job throughput."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
        m = bench.max_over_ranks(ms, world)
        steps, streams = 20, 64
        value = streams * world * steps / (m / 1e3)
        out[rank] = (m, value)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0][0] == out[1][0] == pytest.approx(15.0)
    assert out[0][1] == out[1][1] == pytest.approx(64 * 2 * 20 / 0.015)
