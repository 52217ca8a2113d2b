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


def _place_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from natureuserinterfacestudio_b200.placement import Placement, place_round
        GB = 1 << 30
        pl = Placement([10 * GB, 10 * GB]) if rank == 0 else None
        got, waited = [], []
        # first placement: six streams of 3 GB -> three per GPU, alternating; the seventh waits
        arrivals = [(i, 3 * GB) for i in range(7)]
        mine, waiting = place_round(pl, arrivals, [], rank, world)
        got.append(mine)
        waited.append(waiting)
        # second placement: stream 0 leaves; the waiting stream takes its place
        mine, waiting = place_round(pl, [(6, 3 * GB)], [0], rank, world)
        got.append(mine)
        waited.append(waiting)
        out[rank] = (got, waited)
    finally:
        dist.destroy_process_group()


def test_streams_placed_on_gpus_by_budget_gloo_world2():
    """Sessions -> GPUs at admission: rank 0 places each arriving stream on the GPU with the
    most free HBM budget that holds it, broadcasts the decisions, and every rank admits
    exactly its own streams; a stream that fits nowhere waits until one leaves."""
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_place_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    (g0, w0), (g1, w1) = out[0], out[1]
    assert w0 == w1 == [[6], []]
    assert sorted(g0[0] + g1[0]) == list(range(6)) and len(g0[0]) == len(g1[0]) == 3
    assert not set(g0[0]) & set(g1[0])
    gpu_of_0 = 0 if 0 in g0[0] else 1
    assert (g0 if gpu_of_0 == 0 else g1)[1] == [6] and (g1 if gpu_of_0 == 0 else g0)[1] == []
