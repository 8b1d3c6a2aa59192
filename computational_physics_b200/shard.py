"""Partition of independent lattices (the batched mix) or jobs (the serving queue) across ranks.

Lattices and jobs are independent Markov chains, so a job of many of them shards with no data
exchange at all: every item lives on exactly one rank (one GPU), each rank sweeps its share with
its own batched engine, and only host-side results (per-lattice observables) travel, gathered on
rank 0 over the control plane.  The reference keeps one GPU per process
(utility/execution/hip_context.hpp:24-27, group size 1); this module is what lets one job use
several.

The partition balances device memory: items are placed largest first onto the rank with the
least bytes so far (longest-processing-time greedy), with the bytes of an item the batched
engine's own admission estimate (swb_batch_lattice_bytes), which is proportional to its sites.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Sequence

from ._native import check, lib

__all__ = ["lattice_bytes", "partition", "imbalance", "shard_of", "gather_results"]


def lattice_bytes(L0: int, L1: int, tile: tuple[int, int], lcg_width: int = 16) -> int:
    """Device bytes the batched engine reserves for one lattice (host-side arithmetic, no GPU)."""
    out = ctypes.c_uint64()
    check(lib().swb_batch_lattice_bytes(L0, L1, tile[0], tile[1], lcg_width, ctypes.byref(out)))
    return int(out.value)


def partition(weights: Sequence[int], world: int) -> list[list[int]]:
    """Item indices per rank: heaviest item first onto the lightest rank (ties: lower rank,
    lower index), so every item is placed exactly once and the heaviest rank carries at most
    the lightest rank's load plus one item."""
    if world < 1:
        raise ValueError("world must be >= 1")
    parts: list[list[int]] = [[] for _ in range(world)]
    load = [0] * world
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += weights[i]
    for p in parts:
        p.sort()
    return parts


def imbalance(parts: Sequence[Sequence[int]], weights: Sequence[int]) -> float:
    """Heaviest rank's load over the mean load (1.0 = perfectly balanced)."""
    loads = [sum(weights[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0


def shard_of(weights: Sequence[int], world: int, rank: int) -> list[int]:
    """This rank's item indices."""
    return partition(weights, world)[rank]


def gather_results(local: dict, gather: Callable[[dict], list[dict] | None]) -> dict | None:
    """Merges per-rank {item index: result} dicts on the rank where `gather` returns the list of
    all ranks' dicts (torch.distributed.gather_object on rank 0, or the identity in one
    process); None elsewhere.  Raises if an item was reported twice."""
    parts = gather(local)
    if parts is None:
        return None
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"item {k} reported by two ranks")
            merged[k] = v
    return merged
