"""Multi-GPU work distribution for batches of independent tests.

One LL/PRP test is a strict chain of squarings, so GPUs share work by test, not
inside one transform: each rank (one process per GPU) runs its own batch engine
(lnt_batch) over a cost-balanced share of the work list, and the only exchange
is a host-side gather of results.  The reference runs one test per process on
one GPU (main_process.cu:64-160); there is no reference counterpart to mirror.

Everything here is host logic over torch.distributed (NCCL or gloo), so the
tests run it on CPU with gloo ranks.
"""
from __future__ import annotations

import heapq
import math


def test_cost(exponent: int, iterations: int | None = None, prp: bool = False) -> float:
    """Relative device time of one test: squarings x n log n (n: policy length)."""
    if iterations is None:
        iterations = exponent if prp else exponent - 2
    log_n = max(1, math.ceil(math.log2(max(2, exponent / 32))))  # close to the length policy
    n = 1 << log_n
    return float(iterations) * n * log_n


def partition_by_cost(items: list, world: int, cost=None) -> list[list]:
    """Longest-processing-time split of `items` over `world` ranks: each item
    goes to the currently least loaded rank, heaviest first.  Deterministic, so
    every rank computes the same split without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = cost or (lambda q: test_cost(q))
    order = sorted(range(len(items)), key=lambda i: (-cost(items[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares: list[list] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(items[i])
        heapq.heappush(heap, (load + cost(items[i]), r))
    return shares


def max_over_ranks(value: float, dist=None) -> float:
    """The slowest rank's time (every multi-GPU time is the max over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, float(value))
    return max(out)


def gather_results(local: list, dist=None) -> list:
    """All ranks' result records, concatenated in rank order."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(local))
    return [r for part in out for r in part]
