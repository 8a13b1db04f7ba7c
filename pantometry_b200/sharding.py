"""Ensembles over several GPUs: one process per GPU, each owning a share of the blocks.

The blocks of an ensemble are independent (`Ensemble::run`, crates/pantometry-core/src/
ensemble.rs:102-140), so they shard with no data-path collective: blocks go to ranks by greedy
bin packing on cell count, every rank steps its own share, and the only exchange is one gather
of the per-block FP64 ledgers at the end, put back in block order on the host. The order of the
blocks, not of the ranks, decides every result, as `Ensemble::blocks` requires of its sums
(ensemble.rs:180-230).
"""
from __future__ import annotations

import heapq


def partition(sizes, world):
    """Block indices per rank: largest blocks first, each onto the least-loaded rank (the lower
    rank on a tie); each rank's list in ascending block order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    order = sorted(range(len(sizes)), key=lambda g: (-int(sizes[g]), g))
    for g in order:
        load, r = heapq.heappop(heap)
        shares[r].append(g)
        heapq.heappush(heap, (load + int(sizes[g]), r))
    return [sorted(s) for s in shares]


def gather_ledgers(local, share, count, dist=None):
    """Every rank's per-block ledgers back in block order (on every rank). `local[q]` is the
    ledger of block `share[q]`; without a process group the local list is the whole ensemble."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        pairs = [list(zip(share, local))]
    else:
        pairs = [None] * dist.get_world_size()
        dist.all_gather_object(pairs, list(zip(share, local)))
    out = [None] * count
    for rank_pairs in pairs:
        for g, led in rank_pairs:
            if out[g] is not None:
                raise RuntimeError(f"block {g} was stepped by two ranks")
            out[g] = led
    missing = [g for g, led in enumerate(out) if led is None]
    if missing:
        raise RuntimeError(f"blocks {missing[:8]} were stepped by no rank")
    return out
