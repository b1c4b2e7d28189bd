"""Several GPUs: independent Lucas-Lehmer tests, one process per GPU (replicas only).

A Lucas-Lehmer test is a strict chain of squarings (s_{k+1} = s_k^2 - 2 mod 2^p - 1), so one test
never spans GPUs. A range of exponents splits into independent tests. Each rank takes a share
balanced by squaring cost and runs its tests on its own GPU, and the host gathers the verdicts.
This is the reference's own split of a range over worker threads (PerfNumMultiCLL.py runs
test_one over a thread pool), here across processes. No collective touches the data path. The
only collectives are the device-time maximum and the result gather, both over torch.distributed
(NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
import math


def squaring_cost(p: int) -> float:
    """Relative cost of a whole test of p: (p - 2) squarings of a length-N transform,
    N log2 N each, with N the power of two at <= 18 bits per digit."""
    if p < 3:
        return 0.0
    n = 1 << max(5, math.ceil(math.log2(p / 18.0)))
    return (p - 2) * n * math.log2(n)


def shard(ps, rank: int, world: int):
    """The exponents rank `rank` of `world` tests: greedy largest-first onto the least-loaded
    rank (ties to the lowest rank), so every rank computes the same split without talking."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    load = [(0.0, r) for r in range(world)]
    heapq.heapify(load)
    mine = []
    for p in sorted(ps, key=lambda q: (-squaring_cost(q), q)):
        c, r = heapq.heappop(load)
        if r == rank:
            mine.append(p)
        heapq.heappush(load, (c + squaring_cost(p), r))
    return sorted(mine)


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _world():
    import torch.distributed as dist
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def reduce_max(x: float) -> float:
    """Maximum of x over the ranks (the job's time is its slowest rank's)."""
    if _world() == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float) -> float:
    if _world() == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather(results):
    """Every rank's result list, concatenated and sorted by exponent (on every rank)."""
    if _world() == 1:
        return sorted(results, key=lambda r: r["p"])
    import torch.distributed as dist
    parts = [None] * _world()
    dist.all_gather_object(parts, list(results))
    return sorted((r for part in parts for r in part), key=lambda r: r["p"])
