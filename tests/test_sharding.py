"""Ensemble sharding across ranks (host logic, CPU only): greedy bin packing, and a world-size-2
`gloo` run whose gathered per-block ledgers equal the single-process ones in block order.

The blocks are stepped by the oracle here (no GPU): what is under test is who steps which block
and how the ledgers come back, which is the same for the GPU ranks of `bench.py --gpus N`.
"""
import math
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pantometry_b200 import sharding


def test_partition_is_greedy_balanced_and_complete():
    sizes = [5, 9, 1, 9, 4, 4, 7, 2]
    shares = sharding.partition(sizes, 3)
    assert sorted(g for s in shares for g in s) == list(range(len(sizes)))
    loads = [sum(sizes[g] for g in s) for s in shares]
    assert max(loads) - min(loads) <= max(sizes)
    assert all(s == sorted(s) for s in shares)
    assert sharding.partition(sizes, 3) == shares  # deterministic
    assert sharding.partition(sizes, 1) == [list(range(len(sizes)))]
    assert sharding.partition([], 2) == [[], []]


def test_gather_refuses_double_and_missing_blocks():
    assert sharding.gather_ledgers(["a", "b"], [1, 0], 2) == ["b", "a"]
    with pytest.raises(RuntimeError):
        sharding.gather_ledgers(["a"], [0], 2)


def _blocks():
    from pantometry_b200 import workloads as W

    cfg = W.heat_ensemble(count=7, lo=3, hi=9)
    return cfg["grids"]


def _ledgers_of(indices):
    import oracle
    from pantometry_b200 import workloads as W

    grids = _blocks()
    out = []
    for g in indices:
        src = grids[g]
        nx, ny, nz = src["counts"]
        dx, s = src["dx"], src["substance"]
        o = oracle.Heat((nx, ny, nz), dx, s["density"], s["conductivity"], s["specific_heat"], src["initial"])
        areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
        for f in range(6):
            o.losing_from(f, src["initial"], math.inf, areas[f])
        o.cells = W.ensemble_cells(src)
        assert o.step(0.9 * o.max_stable_dt(), 20) is None
        led = o.ledger()
        out.append((led["total"], led["stored"], led["lost"]))
    return out


def _rank(rank, world, port, result):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grids = _blocks()
        sizes = [int(np.prod(g["counts"])) for g in grids]
        share = sharding.partition(sizes, world)[rank]
        gathered = sharding.gather_ledgers(_ledgers_of(share), share, len(grids), dist)
        if rank == 0:
            result.put(gathered)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_single_process_ledgers():
    ctx = mp.get_context("spawn")
    result = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, result)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = result.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = _ledgers_of(range(len(_blocks())))
    assert gathered == want  # bit for bit, in block order
