"""The multi-GPU form is replicas only: each rank runs its own pool and the
ranks meet only for timing.  This covers that host logic with two gloo
ranks on the CPU: the slowest rank's time is taken, and the whole-job rate
counts every rank's work; the reference arm runs on rank 0 alone."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r took (r + 1) seconds and saw r errors
        got = bench.reduce_max_over_ranks(torch, [float(rank + 1), float(rank)], world, "cpu")
        dist.barrier()
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        assert out[0] == out[1] == [2.0, 1.0]
    # every rank processed 327,680 pairs in at most 2 s
    assert bench.replica_throughput(327680, world, 2.0) == pytest.approx(327680.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        steps, warmup = 1, 3

    assert bench.main_reference(Args()) is None
    assert capsys.readouterr().out == ""
