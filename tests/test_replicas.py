"""The replica logic of the multi-GPU bench (one independent batch of systems per rank), on two
gloo ranks on the CPU: disjoint seeds, the max-over-ranks time, the whole-job rate."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        seeds = bench.replica_seeds(rank, 4)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        local = 1.5 + rank  # rank 1 is the slowest
        slowest = bench.max_over_ranks(local, dist, torch.device("cpu"))
        rate = bench.whole_job_rate(world, 4, 3, slowest)
        out.put((rank, gathered, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, slowest, rate in results:
        flat = [s for seeds in gathered for s in seeds]
        assert len(set(flat)) == len(flat) == 8  # disjoint systems across replicas
        assert slowest == pytest.approx(2.5)     # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 4 * 3 / 2.5)


def test_single_process_helpers():
    import bench

    assert bench.replica_seeds(0, 3) == [0, 1, 2]
    assert bench.max_over_ranks(1.25, None, None) == 1.25
    assert bench.whole_job_rate(1, 32, 3, 2.0) == pytest.approx(48.0)


def test_profile_traffic_reads_the_committed_summary():
    """The bench's roofline traffic comes from the committed ncu summary (keys hold an '=' themselves)."""
    import bench

    for key in ("f32x4,batch=128", "f32x4,batch=64", "f32x4,batch=32", "f64x2,batch=1", "f32,batch=32", "f64,batch=1"):
        value = bench._profile_traffic(key)
        assert value is not None and value > 1e6, key
    assert bench._profile_traffic("f32,batch=7") is None
