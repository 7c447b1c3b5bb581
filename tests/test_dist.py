"""Multi-GPU replicas, on CPU: two gloo ranks run bench.py's rank combination (max of step
times over ranks, sum of work) and its reference-arm rule (rank 0 alone prints)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        times, counts = bench.combine_ranks(dist, [10.0 + rank, 5.0 - rank], [100 * (rank + 1), 7], "cpu")
        out[rank] = (times, counts)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_combine_max_time_and_summed_work():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    for r in range(world):
        times, counts = out[r]
        assert times == [11.0, 5.0]          # slowest rank per entry
        assert counts == [300, 14]           # work of all ranks


def test_single_process_combine_is_identity():
    import bench
    assert bench.combine_ranks(None, [1.5], [3], "cpu") == ([1.5], [3])


def test_reference_arm_prints_on_rank_zero_only(capsys):
    import bench

    class A:
        workload, seed, warmup, steps, gpus = "cfg1", 1, 0, 1, 2
    bench.run_reference_arm(A, 2, 1)       # rank 1: no work, no output
    assert capsys.readouterr().out == ""
