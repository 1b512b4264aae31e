"""The bench's multi-rank path on CPU (gloo, world size 2): replicas get their
own frames, time as the maximum over ranks, and meet at barriers."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench

    r, w, _ = bench.dist_setup("gloo")
    try:
        bench.barrier(w)
        out[r] = (bench.max_over_ranks(10.0 + r, w), tuple(bench.frame_seeds(r, 3)))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_distinct_frames():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 11.0
    assert set(out[0][1]).isdisjoint(out[1][1])


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    class A:
        config = "small"
        steps = 1
        warmup = 0

    assert bench.run_reference(A, rank=1, world=2) is None
