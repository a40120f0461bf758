"""Sharding a laser sweep of independent solves across ranks (one GPU each).

A sweep (many solves of uneven band count and k grid under different pulses)
has no exchange step: every solve is independent.  It is partitioned across
ranks by predicted cost -- longest-processing-time first onto the least
loaded rank -- with no data-path collective; the ranks meet only at the end,
where the host gathers each solve's observables (`gather`, a
torch.distributed object gather over whatever backend the group uses).

The cost of a solve per RK4 step is the algorithmic HBM traffic of its
kernels, which bounds them: (34 + 4 d_E) S bytes for the independent-particle
right-hand side, S = Nk nb^2 16 bytes (the reference counterpart is the k-pool
split of fftPair.cpp:46-57, which divides one solve; here whole solves are
dealt out).
"""
from __future__ import annotations

import heapq


def solve_cost(spec: dict, d_E: int = 2) -> float:
    """Predicted bytes per RK4 step of one sweep solve (workloads.sweep_specs entry)."""
    S = spec["N"] ** 2 * spec["nb"] ** 2 * 16.0
    return (34.0 + 4.0 * d_E) * S


def partition(specs: list[dict], world: int, cost=solve_cost) -> list[list[int]]:
    """Solve indices per rank: LPT (largest cost first onto the least loaded
    rank; ties to the lower rank).  Deterministic for a given input."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(specs)), key=lambda i: (-cost(specs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + cost(specs[i]), r))
    for r in range(world):
        out[r].sort()
    return out


def loads(specs: list[dict], parts: list[list[int]], cost=solve_cost) -> list[float]:
    return [sum(cost(specs[i]) for i in p) for p in parts]


def gather(local: dict, world: int) -> dict:
    """Merge every rank's {solve index: result} on all ranks (host objects,
    after the propagation; torch.distributed must be initialised for world > 1)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts: list = [None] * world
    dist.all_gather_object(parts, local)
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"solve {k} was propagated on two ranks")
            merged[k] = v
    return merged
