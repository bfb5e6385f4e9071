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


def _ladder():
    """Padded orders for grouping: multiples of 32 growing by about 20 %."""
    out, v = [], 64
    while v <= 8192:
        out.append(v)
        v = -(-int(v * 1.2) // 32) * 32
    return out


LADDER = _ladder()


def padded_order(n):
    """The smallest ladder order >= n (multiples of 64 beyond the ladder)."""
    for v in LADDER:
        if v >= n:
            return v
    return -(-int(n) // 64) * 64


def group_plan(orders, n_k, budget_bytes, bytes_per_matrix):
    """Groups of structure indices sharing one padded order: [(nb, [i, ...])].
    Members are in index order; a group holds at most 65535 matrices and
    ``budget_bytes`` of ``bytes_per_matrix(nb)`` each."""
    buckets = {}
    for i, n in enumerate(orders):
        buckets.setdefault(padded_order(n), []).append(i)
    plan = []
    for nb in sorted(buckets):
        per = max(1, int(n_k) * int(bytes_per_matrix(nb)))
        cap = max(1, min(65535 // max(1, int(n_k)), int(budget_bytes // per)))
        idx = buckets[nb]
        for c in range(0, len(idx), cap):
            plan.append((nb, idx[c : c + cap]))
    return plan


class _Ports:
    """The right-hand sides ([B | A^T], B, A) of a group's members, read
    once every member's preparation has finished (after its fills were
    issued)."""

    def __init__(self, ports, ids):
        self._ports, self._ids = ports, ids

    def __iter__(self):
        return (self._ports[i] for i in self._ids)


def _group_bytes(count, nb, P):
    """Device bytes of one group's Z, Z32 and solver workspace (each part
    256-byte aligned), the arena ``_solve_group`` carves them from."""
    from . import _lib

    al = lambda x: (int(x) + 255) & ~255  # noqa: E731
    wsb = _lib.load().mw_zgesv_mixed_batched_workspace_size(nb, P, count)
    return al(count * nb * nb * 16) + al(count * nb * nb * 8) + al(wsb)


def _solve_group(solvers, nb, ks, stream, pw=None, Bs=None, arena=None, wait=None):
    """Batched mixed solve of several structures at the frequencies ks in
    one factorisation: each structure's n x n matrices are filled into the
    leading block of order-nb matrices padded with the identity
    (mw_pad_identity), so every (structure, frequency) system is one matrix
    of one batch.  Returns ({position: Y stack (n_k, P, P)}, iterations)."""
    import ctypes as C

    import torch

    from . import _lib

    lib = _lib.load()
    dev = solvers[0]._torch_device()
    nk = len(ks)
    G = len(solvers)
    count = G * nk
    # right-hand sides per structure: ports plus its KCL rows (Schur step after)
    P = max(s._port_count() + s._kcl_rows_left() for s in solvers)
    wsb = lib.mw_zgesv_mixed_batched_workspace_size(nb, P, count)
    if arena is not None and arena.numel() >= _group_bytes(count, nb, P):
        # views of one allocation made for the whole sweep (no allocation
        # per group)
        al = lambda x: (int(x) + 255) & ~255  # noqa: E731
        o1 = al(count * nb * nb * 16)
        o2 = o1 + al(count * nb * nb * 8)
        Z = arena[: count * nb * nb * 16].view(torch.complex128).view(count, nb, nb)
        Z32 = arena[o1 : o1 + count * nb * nb * 8].view(torch.complex64).view(count, nb, nb)
        ws = arena[o2 : o2 + wsb]
    else:
        Z = torch.empty((count, nb, nb), dtype=torch.complex128, device=dev)
        Z32 = torch.empty((count, nb, nb), dtype=torch.complex64, device=dev)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    k_dev = solvers[0]._upload_k(ks)
    for g, s in enumerate(solvers):
        if wait is not None:
            wait(g)  # this structure's host tables (later ones may still be in preparation)
        n = s._basis().n
        zb, z32b = Z[g * nk : (g + 1) * nk], Z32[g * nk : (g + 1) * nk]
        s._fill_batched(ks, stream, Z=zb, Z32=z32b, ld=nb, k_dev=k_dev)
        _lib.call("mw_pad_identity", n, nb, nk, zb.data_ptr(), nb, nb * nb, z32b.data_ptr(), nb, nb * nb, stream)
    if Bs is None:
        Bs = [s._sweep_rhs() for s in solvers]
    Bs = list(Bs)  # (R = [B | A^T], B, A) per structure
    # the right-hand sides of every structure, staged in page-locked memory
    # and uploaded with one stream-ordered copy (pageable uploads would make
    # the host wait for the fills queued before them)
    Bh = torch.zeros((G, P, nb), dtype=torch.complex128, pin_memory=True)
    for g, (R, _B, _A) in enumerate(Bs):
        Bh[g, : R.shape[1], : R.shape[0]] = torch.from_numpy(np.ascontiguousarray(R.T))
    Bg = Bh.to(dev, non_blocking=True)
    Bd = Bg.repeat_interleave(nk, dim=0)
    if pw is None:
        pw = _group_width(solvers[0], nb, Z, Z32, Bd, P, stream)
    X = torch.empty((count, P, nb), dtype=torch.complex128, device=dev)
    ipiv = torch.empty((count, nb), dtype=torch.int32, device=dev)
    info = torch.zeros(count, dtype=torch.int32, device=dev)
    it, corr = C.c_int32(0), C.c_double(0.0)
    s0 = solvers[0]
    _lib.call("mw_zgesv_mixed_batched", nb, P, count, int(pw), Z.data_ptr(), nb, nb * nb, Z32.data_ptr(), nb,
              nb * nb, ipiv.data_ptr(), info.data_ptr(), Bd.data_ptr(), nb, P * nb, X.data_ptr(),
              float(s0.mixed_tol), int(s0.mixed_max_iter), ws.data_ptr(), wsb, C.byref(it), C.byref(corr), stream)
    Xh = X.cpu().numpy()
    out = {}
    from .bspline import _swept_y

    for g, (R, B, A) in enumerate(Bs):
        n, m = R.shape
        out[g] = _swept_y(Xh[g * nk : (g + 1) * nk, :m, :n], B, A)
    return out, int(it.value)


def _group_width(s0, nb, Z, Z32, Bd, P, stream):
    """Panel width for padded order nb: the autotuner's cached choice, else
    timed on up to 64 matrices of this group (their complex64 copies are
    factored in scratch buffers)."""
    import ctypes as C

    import torch

    from . import _lib, autotune

    lib = _lib.load()
    m = min(Z.shape[0], 64)

    def time_width(w):
        z32 = Z32[:m].clone()
        X = torch.empty((m, P, nb), dtype=torch.complex128, device=Z.device)
        ipiv = torch.empty((m, nb), dtype=torch.int32, device=Z.device)
        info = torch.zeros(m, dtype=torch.int32, device=Z.device)
        wsb = lib.mw_zgesv_mixed_batched_workspace_size(nb, P, m)
        ws = torch.empty(wsb, dtype=torch.uint8, device=Z.device)
        st = torch.cuda.current_stream(Z.device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _rep in range(2):  # the first run warms up
            z32.copy_(Z32[:m])
            it, corr = C.c_int32(0), C.c_double(0.0)
            a.record(st)
            _lib.call("mw_zgesv_mixed_batched", nb, P, m, int(w), Z.data_ptr(), nb, nb * nb, z32.data_ptr(), nb,
                      nb * nb, ipiv.data_ptr(), info.data_ptr(), Bd.data_ptr(), nb, P * nb, X.data_ptr(),
                      float(s0.mixed_tol), int(s0.mixed_max_iter), ws.data_ptr(), wsb, C.byref(it),
                      C.byref(corr), stream)
            b.record(st)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return ms[-1]

    return autotune.choose(nb, 0, "grouped", time_width)


def shard_indices(structs, rank, world):
    """This rank's structures: the LPT partition of ``structure_cost``."""
    return partition([structure_cost(kw) for kw in structs], world)[rank]


class _DeviceGroups:
    """Solves the groups of a sweep on the GPU: one device arena for every
    group, the heaviest groups first, and a helper thread that builds the
    next structures' host tables (packed for one upload each) while the
    current group is filled and factorised."""

    def __init__(self, solvers, ks, plan_ids, P_max):
        import concurrent.futures as cf

        import torch

        self.solvers, self.ks = solvers, ks
        first = solvers[plan_ids[0][1][0]]
        self.dev = first._torch_device()
        self.stream = torch.cuda.current_stream(self.dev).cuda_stream
        self.arena = torch.empty(max(_group_bytes(len(ids) * len(ks), nb, P_max) for nb, ids in plan_ids),
                                 dtype=torch.uint8, device=self.dev)
        self.ports = {}
        self.ex = cf.ThreadPoolExecutor(max_workers=1)
        self.futs = {i: self.ex.submit(self._prep, i) for _nb, ids in plan_ids for i in ids}

    def _prep(self, i):
        # host work only (tables packed for one upload, port columns); the
        # uploads themselves are stream-ordered on the main thread, so the
        # helper never waits for the device
        s = self.solvers[i]
        s._packed_tables()
        if s._loading is not None:
            s._loading_tables()
        self.ports[i] = s._sweep_rhs()

    def solve(self, nb, ids):
        def wait(g):
            self.futs[ids[g]].result()

        res, _it = _solve_group([self.solvers[i] for i in ids], nb, self.ks, self.stream, arena=self.arena,
                                wait=wait, Bs=_Ports(self.ports, ids))
        return res

    def single(self, solver):
        return solver.compute_y_matrix_swept(self.ks)

    def close(self):
        self.ex.shutdown(wait=True)


def grouped_mixed_sweep(structs, ks, device=None, budget_bytes=32 << 30, indices=None, groups=None):
    """{index: (n_k, P, P) Y stack} for the given structures, every one at
    the frequencies ks, through grouped batched solves: structures are
    bucketed by padded order (``padded_order``), and each group's
    (structure, frequency) systems are filled into one padded stack and
    factorised by one batched mixed-precision solve.  Structures the batched
    route does not serve (finite grounds, KCL constraint rows, orders above
    the batched panel's limit) take their own ``compute_y_matrix_swept``.

    ``groups(solvers, ks, plan, P_max)`` makes the group solver (``solve(nb,
    ids)`` -> {position: Y stack}, ``single(solver)``, ``close()``); the
    default solves on the GPU."""
    import momwire_b200

    from . import _lib

    indices = list(range(len(structs))) if indices is None else list(indices)
    solvers = {i: momwire_b200.BSplineSolver(**structs[i], precision="mixed", device=device) for i in indices}
    ks = np.asarray(ks, dtype=np.float64)
    grouped, single = [], []
    for i in indices:
        s = solvers[i]
        (grouped if s._swept_batched_available() and padded_order(s._basis_count()) <= 1600 else single).append(i)
    if groups is None:
        lib = _lib.load()

        def per_matrix(nb):
            return nb * nb * 24 + lib.mw_zgesv_mixed_batched_workspace_size(nb, 1, 1) + nb * 64

        groups = _DeviceGroups
    else:
        def per_matrix(nb):
            return nb * nb * 24

    plan = group_plan([solvers[i]._basis_count() for i in grouped], len(ks), budget_bytes, per_matrix)
    # the heaviest groups first: the first group waits for its host tables,
    # after which the helper prepares the rest while the GPU works
    plan.sort(key=lambda g: -len(g[1]) * g[0] ** 3)
    plan_ids = [(nb, [grouped[j] for j in members]) for nb, members in plan]
    out = {}
    if not plan_ids and not single:
        return out
    P_max = max([solvers[i]._port_count() + solvers[i]._kcl_rows_left() for i in grouped] or [1])
    runner = groups(solvers, ks, plan_ids, P_max) if plan_ids else None
    try:
        for i in single:
            out[i] = runner.single(solvers[i]) if runner is not None else solvers[i].compute_y_matrix_swept(ks)
        for nb, ids in plan_ids:
            res = runner.solve(nb, ids)
            for g, i in enumerate(ids):
                out[i] = res[g]
    finally:
        if runner is not None:
            runner.close()
    return {i: out[i] for i in indices}


def mixed_sweep_fn(device=None):
    """solve_fn for ``solve_shard``: the batched mixed-precision sweep of one
    structure on this rank's GPU."""
    import momwire_b200

    def fn(kw, ks):
        return momwire_b200.BSplineSolver(**kw, precision="mixed", device=device).compute_y_matrix_swept(ks)

    return fn
