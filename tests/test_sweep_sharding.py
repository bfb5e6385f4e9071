"""Sharding of multi-structure sweeps over ranks: the LPT partition and the
gather of per-structure results, run as two gloo ranks on the CPU (the
solve is a stand-in; the GPU sweep itself is covered by the gpu tests)."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from momwire_b200 import sweep
from momwire_b200.workloads import yagi_sweep


def test_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 100, 37) ** 3
    parts = sweep.partition(costs, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(37))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()  # LPT bound
    assert sweep.partition([5.0], 3) == [[0], [], []]


def test_structure_cost_counts_segments():
    structs, _ks = yagi_sweep(n_structures=3, n_freq=4, seed=0)
    for kw in structs:
        assert sweep.structure_cost(kw) == float(sum(kw["n_per_edge_per_wire"])) ** 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    structs, ks = yagi_sweep(n_structures=9, n_freq=3, seed=1)
    parts = sweep.partition([sweep.structure_cost(s) for s in structs], world)
    fake = lambda kw, k: np.full((len(k), 1, 1), sum(kw["n_per_edge_per_wire"]) + 1j * len(kw["wires"]))  # noqa: E731
    local = sweep.solve_shard(structs, ks, parts[rank], fake)
    merged = sweep.gather(local)
    if rank == 0:
        out.put({i: complex(v[0, 0, 0]) for i, v in merged.items()})
    dist.destroy_process_group()


def test_two_rank_gather_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    structs, _ks = yagi_sweep(n_structures=9, n_freq=3, seed=1)
    want = {i: complex(sum(kw["n_per_edge_per_wire"]), len(kw["wires"])) for i, kw in enumerate(structs)}
    assert got == want


class _FakeGroups:
    """Stand-in group solver (no GPU): each structure's Y stack is filled
    with (segments + 1j * wires), tagged with the padded order it was
    grouped at, so that the test can check both the routing and the merge."""

    log = []

    def __init__(self, solvers, ks, plan, P_max):
        self.solvers, self.ks = solvers, ks

    def _y(self, s, tag):
        kw_segs = sum(sum(npe) for npe in s.n_per_edge_per_wire)
        return np.full((len(self.ks), 1, 1), kw_segs + 1j * len(s.wires_polylines) + 1000 * tag)

    def solve(self, nb, ids):
        _FakeGroups.log.append((nb, list(ids)))
        return {g: self._y(self.solvers[i], sweep.padded_order(self.solvers[i]._basis_count()) == nb)
                for g, i in enumerate(ids)}

    def single(self, solver):
        return self._y(solver, 0)

    def close(self):
        pass


def _grouped_rank(rank, world, port, out):
    """The bench's shard path on one gloo rank: this rank's LPT share,
    ``grouped_mixed_sweep(indices=...)`` with a stand-in group solver, and
    the rank-0 merge."""
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    structs, ks = yagi_sweep(n_structures=11, n_freq=3, seed=2)
    idx = sweep.shard_indices(structs, rank, world)
    local = sweep.grouped_mixed_sweep(structs, ks, indices=idx, groups=_FakeGroups)
    assert sorted(local) == sorted(idx)
    merged = sweep.gather(local)
    if rank == 0:
        out.put({i: complex(v[0, 0, 0]) for i, v in merged.items()})
    dist.destroy_process_group()


def test_two_rank_grouped_sweep_shards_and_merges():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grouped_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    structs, _ks = yagi_sweep(n_structures=11, n_freq=3, seed=2)
    # every structure once, grouped at its own padded order (tag 1000)
    want = {i: complex(sum(kw["n_per_edge_per_wire"]) + 1000, len(kw["wires"])) for i, kw in enumerate(structs)}
    assert got == want


def test_grouped_sweep_groups_by_padded_order_single_rank():
    structs, ks = yagi_sweep(n_structures=7, n_freq=2, seed=3)
    _FakeGroups.log = []
    out = sweep.grouped_mixed_sweep(structs, ks, groups=_FakeGroups)
    assert sorted(out) == list(range(7))
    seen = sorted(i for _nb, ids in _FakeGroups.log for i in ids)
    assert seen == list(range(7))
    # groups in decreasing work order, one padded order each
    work = [len(ids) * nb ** 3 for nb, ids in _FakeGroups.log]
    assert work == sorted(work, reverse=True)


def test_padded_order_ladder():
    """Padded orders are multiples of 32, at most ~20 % above n, monotone."""
    prev = 0
    for n in range(1, 3000, 7):
        nb = sweep.padded_order(n)
        assert nb >= n and nb % 32 == 0 and nb >= prev
        assert nb <= max(64, int(n * 1.2) + 64)
        prev = nb


def test_group_plan_caps_memory_and_batch():
    orders = [40, 60, 500, 470, 481, 1000, 990, 65]
    plan = sweep.group_plan(orders, 64, budget_bytes=3 * 64 * 480 * 480 * 24, bytes_per_matrix=lambda nb: nb * nb * 24)
    seen = sorted(i for _nb, g in plan for i in g)
    assert seen == list(range(len(orders)))
    for nb, g in plan:
        assert all(sweep.padded_order(orders[i]) == nb for i in g)
        assert len(g) * 64 * nb * nb * 24 <= 3 * 64 * 480 * 480 * 24 or len(g) == 1
    # 65535 matrices at most per group
    plan = sweep.group_plan([100] * 2000, 64, budget_bytes=1 << 60, bytes_per_matrix=lambda nb: 1)
    assert all(len(g) * 64 <= 65535 for _nb, g in plan)
    assert sum(len(g) for _nb, g in plan) == 2000
