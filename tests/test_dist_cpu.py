"""The multi-rank (replica) path of bench.py on CPU: world size 2 over gloo,
rendezvous on 127.0.0.1 -- barrier, max-over-ranks timing and the whole-job
aggregate, the same helpers the GPU runs use over NCCL."""

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


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench

    r, w, lr = bench.dist_env()
    bench.init_dist(w, backend="gloo")
    try:
        bench.barrier(w)
        ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        mx = bench.max_over_ranks(ms, w)
        value = bench.aggregate_value(1e9, w, mx)
        q.put((r, w, lr, mx, value))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_gloo_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for r, (rank, w, lr, mx, value) in enumerate(got):
        assert (rank, w, lr) == (r, world, r)
        assert mx == 15.0  # max over ranks, not the local time
        assert value == pytest.approx(2 * 1e9 / 0.015 / 1e9)  # units of both ranks over the slowest time
