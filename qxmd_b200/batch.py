"""Independent cells spread over GPUs: one process per GPU, each running its
share of the cells with no exchange on the data path, results gathered on the
host at the end.

The reference parallelises one cell over MPI ranks (bands and G vectors,
S/commwv.f90); a batch of independent cells needs none of that: each cell's
SCF iteration is self-contained, so the cells are partitioned by an estimate
of their cost and every rank advances its own cells.  The only collective is
the gather of the per-cell results (and the max of the timings) after the
timed region.
"""
from __future__ import annotations

import math


def cell_cost(nband: int, grid, nplwex: int) -> float:
    """Relative cost of one SCF iteration of a cell: the band FFTs
    (nband * N log2 N) plus the band-space contractions (nband^2 * nplwex)."""
    n = grid[0] * grid[1] * grid[2]
    return nband * n * math.log2(n) + nband * nband * nplwex


def partition(costs, nranks: int) -> list[list[int]]:
    """Cells to ranks, longest first to the least loaded rank (ties to the
    lower rank, so every process computes the same assignment); each rank's
    list in ascending cell order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * nranks
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def gather_results(local: dict, world: int) -> dict:
    """Per-cell results of every rank, merged on all ranks (torch.distributed
    all_gather_object; a plain copy when world is 1)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, local)
    merged = {}
    for d in out:
        merged.update(d)
    return merged
