"""CPU: the multi-GPU split of a batch (cuda_b200/shard.py), with world_size-2
gloo process groups on 127.0.0.1 standing in for one process per GPU.

Covers: the deterministic cost-balanced partition (every rank computes the
same disjoint cover of the work list), the gather of results and the
max-over-ranks time, and a rank that fails before the gather: the others end
with an error from a short process-group timeout instead of waiting forever.
"""
import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cuda_b200 import shard


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_a_balanced_cover():
    exps = list(range(10007, 10007 + 2 * 500, 2))
    for world in (1, 2, 3, 8):
        shares = shard.partition_by_cost(exps, world)
        flat = [q for s in shares for q in s]
        assert sorted(flat) == sorted(exps) and len(flat) == len(set(flat))
        loads = [sum(shard.test_cost(q) for q in s) for s in shares]
        assert max(loads) <= min(loads) * 1.05 + max(shard.test_cost(q) for q in exps)
    assert shard.partition_by_cost(exps, 4) == shard.partition_by_cost(list(exps), 4)


def _worker(rank, world, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        exps = list(range(100003, 100003 + 2 * 64, 2))
        mine = shard.partition_by_cost(exps, world)[rank]
        if mode == "fail" and rank == 1:
            raise SystemExit(3)  # leaves before the gather, nothing in flight
        results = [{"q": q, "rank": rank} for q in mine]
        allr = shard.gather_results(results, dist)
        t = shard.max_over_ranks(1.0 + rank, dist)
        out.put((rank, sorted(r["q"] for r in allr) == sorted(exps), t))
    except Exception as e:  # the surviving rank reports the failed collective
        out.put((rank, "error", type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
    got = []
    while not q.empty():
        got.append(q.get())
    for p in ps:
        if p.is_alive():
            p.kill()
    return sorted(got, key=lambda g: g[0])


def test_gather_and_max_over_two_gloo_ranks():
    got = _run(2, "ok")
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] is True for g in got)
    assert all(g[2] == 2.0 for g in got)  # the slowest rank's time on every rank


def test_a_failed_rank_ends_the_collective_with_an_error():
    got = _run(2, "fail")
    assert got and got[0][0] == 0 and got[0][1] == "error"
