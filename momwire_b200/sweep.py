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


def solve_shard(structs, ks, indices, solve_fn, workers=1, device=None):
    """{structure index: solve_fn(kw, ks)} over this rank's indices.

    With workers > 1 the structures run on that many host threads, each
    issuing to its own CUDA stream, so that one structure's host work and
    small kernels overlap another's (a batched solve of one structure holds
    only a CTA per matrix during its panels)."""
    if workers <= 1:
        return {i: solve_fn(structs[i], ks) for i in indices}
    import concurrent.futures as cf

    import torch

    dev = torch.device("cuda", device if device is not None else torch.cuda.current_device())
    streams = [torch.cuda.Stream(device=dev) for _ in range(workers)]
    slot = {}

    def run(i):
        import threading

        tid = threading.get_ident()
        if tid not in slot:
            slot[tid] = streams[len(slot) % workers]
        with torch.cuda.device(dev), torch.cuda.stream(slot[tid]):
            out = solve_fn(structs[i], ks)
            torch.cuda.current_stream().synchronize()
        return i, out

    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        res = dict(ex.map(run, indices))
    return {i: res[i] for i in indices}


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
