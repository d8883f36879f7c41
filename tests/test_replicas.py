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


def _scan_costs():
    """The 48 bond-scan systems' costs (grid points: every member takes a similar number of applies)."""
    import bench
    import __graft_entry__

    pkg = __graft_entry__.package()
    shapes = []
    for bond in bench.SCAN_BONDS:
        system = bench.scan_system(bond)
        shapes.append(pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device="cpu").shape)
    return pkg, shapes, [pkg.replicas.system_cost(s) for s in shapes]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_cost_partition_of_the_bond_scan(world):
    """Every system on exactly one rank, each share in index order, the same answer every time, and
    the longest-processing-time bound: no rank above the mean load plus the costliest system."""
    pkg, shapes, costs = _scan_costs()
    assert len(set(shapes)) > 10  # the boxes grow with R: the costs differ
    shares = pkg.replicas.partition_by_cost(costs, world)
    assert len(shares) == world
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(48))
    assert all(s == sorted(s) for s in shares)
    assert shares == pkg.replicas.partition_by_cost(costs, world)
    loads = pkg.replicas.share_loads(costs, shares)
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    if world > 1:  # far better than an equal count of systems in index order
        naive = [list(range(48))[r * 48 // world:(r + 1) * 48 // world] for r in range(world)]
        assert max(loads) < max(pkg.replicas.share_loads(costs, naive))


def test_partition_and_gather_edge_cases():
    import __graft_entry__

    pkg = __graft_entry__.package()
    rep = pkg.replicas
    assert rep.partition_by_cost([], 3) == [[], [], []]
    assert rep.partition_by_cost([5.0, 1.0], 4) == [[0], [1], [], []]
    assert rep.partition_by_cost([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        rep.partition_by_cost([1.0], 0)
    with pytest.raises(ValueError):
        rep.partition_by_cost([-1.0], 2)
    with pytest.raises(ValueError):
        rep.system_cost((4, 0, 4))
    assert rep.gather_by_index({1: "b", 0: "a"}, 2) == ["a", "b"]
    with pytest.raises(ValueError):
        rep.gather_by_index({0: "a"}, 2)


def _scan_rank_main(rank: int, world: int, port: int, out) -> None:
    import datetime

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pkg, shapes, costs = _scan_costs()
        shares = pkg.replicas.partition_by_cost(costs, world)
        agreed = [None] * world
        dist.all_gather_object(agreed, shares)
        # each rank "solves" only its share: a per-system scalar made from the system's own index
        local = {k: {"total": -0.5 - 0.001 * k, "rank": rank} for k in shares[rank]}
        gathered = pkg.replicas.gather_by_index(local, len(costs), dist)
        out.put((rank, agreed, shares, gathered))
    finally:
        dist.destroy_process_group()


def test_scan_partition_and_gather_on_two_gloo_ranks():
    """Two gloo ranks partition the scan alike, each solves a disjoint share, and rank 0 gathers
    every system's result in the original order (the other rank gets None)."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_scan_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, agreed0, shares0, gathered0), (_, agreed1, shares1, gathered1) = results
    assert shares0 == shares1  # each rank's whole partition: the same on both
    assert agreed0 == agreed1 == [shares0, shares0]
    assert gathered1 is None
    assert [g["total"] for g in gathered0] == [-0.5 - 0.001 * k for k in range(48)]
    assert {g["rank"] for g in gathered0} == {0, 1}
    assert all(gathered0[k]["rank"] == r for r in range(world) for k in shares0[r])
