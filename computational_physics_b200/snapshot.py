"""On-disk snapshots of a lattice's Markov-chain state, for preempting and resuming jobs.

The reference keeps no on-disk state.  A snapshot here is one ``.npz`` file with the geometry
(L0, L1, tile, lcg width), the spins (uint8 0/1, [L1, L0]), the per-tile lcg32 streams in
LCG32_State terms (state, a, c: [tiles, W] uint32; iteration: [tiles] uint32), and, when
present, the sweeps done, the recorded (e, m) integer sums and the FP64 accumulators.
Restoring the spins and streams into a lattice of the same geometry continues the chain
bit-identically: ``SwendsenWang2D.restore`` / ``BatchedSW.restore``.
"""
from __future__ import annotations

import numpy as np

_FIELDS = ("spins", "rng_state", "rng_a", "rng_c", "rng_iteration", "samples", "accumulators")


def _npz(path: str) -> str:
    """The file name save() writes and load() reads: ``path`` with ``.npz`` appended unless it
    already ends so (numpy's own rule for np.savez)."""
    return path if path.endswith(".npz") else path + ".npz"


def save(path: str, snap: dict) -> None:
    meta = np.array([snap["L0"], snap["L1"], snap["tile"][0], snap["tile"][1], snap["lcg_width"],
                     snap.get("sweeps_done", 0)], np.int64)
    np.savez(_npz(path), meta=meta, **{k: np.asarray(snap[k]) for k in _FIELDS if k in snap})


def load(path: str) -> dict:
    with np.load(_npz(path)) as f:
        m = f["meta"]
        snap = {"L0": int(m[0]), "L1": int(m[1]), "tile": (int(m[2]), int(m[3])), "lcg_width": int(m[4]),
                "sweeps_done": int(m[5])}
        for k in _FIELDS:
            if k in f:
                snap[k] = f[k]
    if snap["spins"].shape != (snap["L1"], snap["L0"]):
        raise ValueError("snapshot spins do not match its extent")
    W = snap["lcg_width"]
    tiles = (-(-snap["L0"] // snap["tile"][0])) * (-(-snap["L1"] // snap["tile"][1]))
    for k in ("rng_state", "rng_a", "rng_c"):
        if k in snap and snap[k].shape != (tiles, W):
            raise ValueError(f"snapshot {k} has shape {snap[k].shape}, its geometry needs {(tiles, W)}")
    if "rng_iteration" in snap and snap["rng_iteration"].shape != (tiles,):
        raise ValueError(f"snapshot rng_iteration has shape {snap['rng_iteration'].shape}, its geometry needs "
                         f"{(tiles,)}")
    return snap
