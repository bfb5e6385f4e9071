"""Frequency sweeps of many structures, sharded over ranks.

The reference sweeps one structure at a time on the host
(``compute_y_matrix_swept``, ``_port_solution.py:142``; ``bspline.py:4181-4440``).
A sweep over many independent structures has no exchange step until the
results are collected, so it shards with no collective on the data path:

* ``partition`` assigns structures to ranks by longest-processing-time first
  on the n^3 cost of their factorisations (a structure is never split, its
  frequencies share one batched fill and factorisation);
* every rank solves its shard on its own GPU (``BSplineSolver.
  compute_y_matrix_swept``: one batched fill and one batched mixed-precision
  LU per chunk of frequencies);
* ``gather`` collects the (structure index -> Y stack) results on rank 0 with
  one ``gather_object`` (NCCL or gloo).
"""

from __future__ import annotations

import heapq

import numpy as np


def partition(costs, world):
    """Indices of the structures each rank solves: LPT scheduling on the
    given costs (largest first onto the least-loaded rank, ties to the lower
    rank).  Returns a list of ``world`` sorted index lists."""
    costs = np.asarray(costs, dtype=float)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def structure_cost(kw):
    """n^3 of a structure's factorisation, from its segment counts (each
    B-spline basis count is within a few of the segment count)."""
    wires = kw["wires"]
    npe = kw.get("n_per_edge_per_wire")
    nsegs = kw.get("nsegs", 101)
    n = 0
    for w, pl in enumerate(wires):
        edges = len(pl) - 1
        e = npe[w] if npe is not None else None
        if e is None:
            n += nsegs * edges
        elif np.isscalar(e):
            n += int(e) * edges
        else:
            n += int(sum(e))
    return float(n) ** 3


def solve_shard(structs, ks, indices, solve_fn):
    """{structure index: solve_fn(kw, ks)} over this rank's indices."""
    return {i: solve_fn(structs[i], ks) for i in indices}


def gather(local, group=None):
    """Merge every rank's {index: result} on rank 0 (others get None)."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    buf = [None] * world if rank == 0 else None
    dist.gather_object(local, buf, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in buf:
        merged.update(part)
    return merged


def mixed_sweep_fn(device=None):
    """solve_fn for ``solve_shard``: the batched mixed-precision sweep of one
    structure on this rank's GPU."""
    import momwire_b200

    def fn(kw, ks):
        return momwire_b200.BSplineSolver(**kw, precision="mixed", device=device).compute_y_matrix_swept(ks)

    return fn
