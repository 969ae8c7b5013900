"""Host logic of the multi-GPU bench path on two CPU ranks (gloo): situation sharding (weak
scaling, no exchange during the solve), replicas for a single situation, and the max-over-ranks
timing reduction that bench.py applies to device times."""
import os
import socket
import sys

import pytest
import torch.distributed as td
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    from gral_b200 import prep
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sits = bench.rank_situations(None, 144, rank, world)
        keys = sorted((round(s.direction_deg, 6), s.speed_10m) for s in sits)
        gathered = [None] * world
        td.all_gather_object(gathered, keys)
        single = bench.rank_situations(prep.Situation(direction_deg=225.0), 144, rank, world)
        reps = [None] * world
        td.all_gather_object(reps, [(s.direction_deg, s.speed_10m) for s in single])
        t = bench.max_over_ranks(10.0 + rank, None)
        out[rank] = (gathered, reps, t)
    finally:
        td.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharding_and_max_reduction(world):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    assert sorted(out.keys()) == list(range(world))
    gathered, reps, _ = out[0]
    sets = [set(g) for g in gathered]
    assert all(len(s) == 144 for s in sets)                     # fixed work per rank
    assert not (sets[0] & sets[1])                              # disjoint shards
    assert reps[0] == reps[1] == [(225.0, 3.0)]                 # one situation: replicas
    assert all(out[r][2] == 10.0 + world - 1 for r in range(world))   # max over ranks everywhere


def test_rank0_keeps_the_144_situation_set():
    sys.path.insert(0, ROOT)
    import bench
    a = bench.rank_situations(None, 144, 0, 1)
    b = bench.batched_situations(144)
    assert [(x.direction_deg, x.speed_10m, x.obukhov) for x in a] == \
        [(x.direction_deg, x.speed_10m, x.obukhov) for x in b]
    assert sorted({x.speed_10m for x in a}) == [0.5, 1.0, 2.0, 4.0]
    assert len({x.direction_deg for x in a}) == 36


def test_max_over_ranks_without_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
