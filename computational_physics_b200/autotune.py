"""Autotuner for the batched engine: per lattice side L it picks the tile shape (which fixes
how each lcg32 stream is consumed, exactly as the reference's TILE_SIZE_X / TILE_SIZE_Y do on
its CPU path) and the tiles per work item (which fixes how many lcg lanes -- threads -- work
on one block), by timing batched sweeps of many copies of an L x L lattice on the GPU.

Results are cached as JSON per device name and lcg width in ``tuned/``; :func:`choice` reads the
cache and falls back to the nearest tuned L, then to 16 x 8 tiles.

    python -m computational_physics_b200.autotune --sides 64 96 128 192 256 384 512
"""
from __future__ import annotations

import argparse
import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "tuned")

TILES = [(16, 8), (8, 8), (32, 4), (16, 16), (32, 8), (8, 16), (16, 4), (32, 2)]
BLOCKS = [(0, 0), (0, 2), (0, 1), (4, 0), (2, 0)]
DEFAULT = {"tile": [16, 8], "block": [0, 0]}


def device_name(device: int = 0) -> str:
    try:
        import subprocess
        out = subprocess.run(["nvidia-smi", f"--id={device}", "--query-gpu=name", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout.strip()
        return out or "unknown"
    except Exception:
        return "unknown"


def cache_path(name: str, lcg_width: int) -> str:
    slug = re.sub(r"[^a-z0-9]+", "_", name.lower()).strip("_")
    return os.path.join(TUNED, f"{slug}_w{lcg_width}.json")


def load(name: str | None = None, lcg_width: int = 16) -> dict:
    path = cache_path(name or device_name(), lcg_width)
    if not os.path.exists(path):
        # any B200 table is better than none
        cands = [p for p in (os.listdir(TUNED) if os.path.isdir(TUNED) else []) if p.endswith(f"_w{lcg_width}.json")]
        if not cands:
            return {}
        path = os.path.join(TUNED, sorted(cands)[0])
    with open(path) as f:
        return json.load(f)


def choice(L: int, table: dict) -> tuple[tuple[int, int], tuple[int, int]]:
    """(tile, block) for side L: the tuned entry of L, else of the nearest tuned side."""
    entries = table.get("sides", {})
    if not entries:
        return tuple(DEFAULT["tile"]), tuple(DEFAULT["block"])
    key = str(L) if str(L) in entries else min(entries, key=lambda k: abs(int(k) - L))
    e = entries[key]["best"]
    return tuple(e["tile"]), tuple(e["block"])


def time_config(cp, L: int, tile, block, copies: int, rounds: int, lcg_width: int, device: int) -> float:
    """ns per site update of `copies` L x L lattices swept together."""
    with cp.BatchedSW(capacity=copies, lcg_width=lcg_width, device=device) as b:
        for k in range(copies):
            lid = b.add(L, L, 2.2691853, 1 + 7919 * k, tile, block)
            b.hot_start(lid, 1 + k)
        b.sweep(3)
        b.synchronize()
        best = float("inf")
        for _ in range(3):
            ms = float(b.sweep_timed(rounds)[0])
            best = min(best, ms)
    return best * 1e6 / (rounds * copies * L * L)


def tune(sides, lcg_width: int = 16, device: int = 0, target_sites: float = 16e6, rounds: int = 10,
         verbose: bool = True) -> dict:
    import computational_physics_b200 as cp
    name = device_name(device)
    result = {"device": name, "lcg_width": lcg_width, "sides": {}}
    for L in sides:
        copies = int(max(1, min(4096, target_sites // (L * L))))
        trials = []
        for tile in TILES:
            if tile[0] > L or tile[1] > L:
                continue
            seen = set()
            for block in BLOCKS:
                try:
                    with cp.BatchedSW(capacity=1, lcg_width=lcg_width, device=device) as probe:
                        info = probe.info(probe.add(L, L, 2.2691853, 1, tile, block))
                except cp.NativeError:
                    continue
                shape = (info["block_x"], info["block_y"])
                if shape in seen:
                    continue
                seen.add(shape)
                ns = time_config(cp, L, tile, block, copies, rounds, lcg_width, device)
                trials.append({"tile": list(tile), "block": list(shape), "ns_per_site": ns})
                if verbose:
                    print(f"L={L} tile={tile} block={shape} copies={copies}: {ns:.4f} ns/site", flush=True)
        best = min(trials, key=lambda t: t["ns_per_site"])
        result["sides"][str(L)] = {"best": best, "trials": trials, "copies": copies}
    return result


def save(result: dict) -> str:
    os.makedirs(TUNED, exist_ok=True)
    path = cache_path(result["device"], result["lcg_width"])
    with open(path, "w") as f:
        json.dump(result, f, indent=1)
    return path


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--sides", type=int, nargs="+", default=[64, 96, 128, 192, 256, 384, 512])
    ap.add_argument("--lcg-width", type=int, default=16)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    print(save(tune(args.sides, args.lcg_width, args.device)))


if __name__ == "__main__":
    main()
