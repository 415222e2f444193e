"""Spreading independent molecules over ranks (one process per GPU).

Molecules share nothing, so the only multi-rank work is bookkeeping: a longest-processing-time
first partition of the molecules by estimated cost (SCF cost grows as n_AO^3), each rank solving
its share with the batched solver on its own GPU, and one gather of the result records.  There
is no data-path collective.  ``torch.distributed`` carries the gather (NCCL on GPUs; gloo on the
CPU, which is how the tests run it).
"""

from __future__ import annotations

import heapq

import numpy as np


def molecule_cost(numbers) -> float:
    z = np.asarray(numbers).reshape(-1)
    n = float(np.sum(np.where(z == 1, 1, 4)))
    return n ** 3 + 100.0 * n  # eigen/purification work plus a per-molecule floor


def partition(costs, world: int) -> list[list[int]]:
    """LPT: molecules in decreasing cost, each to the currently lightest rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def solve_sharded(mols, solve, dist=None):
    """``mols``: list of (numbers, xyz_bohr, charge, multiplicity); ``solve(list) -> list of
    result dicts``.  Returns every molecule's result, in input order, on every rank."""
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    parts = partition([molecule_cost(m[0]) for m in mols], world)
    mine = parts[rank]
    local = solve([mols[i] for i in mine]) if mine else []
    pairs = list(zip(mine, local))
    if dist:
        gathered = [None] * world
        dist.all_gather_object(gathered, pairs)
    else:
        gathered = [pairs]
    out = [None] * len(mols)
    for chunk in gathered:
        for i, r in chunk:
            out[i] = r
    return out
