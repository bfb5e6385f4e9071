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
