"""A fixed single-lattice workload for profilers (ncu): create, hot start, sweep, exit.

    python -m computational_physics_b200.profile_case --L 8192 --tile 16 8 --sweeps 2

Launch order: k_rng_init, k_hot_start, then per sweep k_assign, k_merge, k_flip.
"""
from __future__ import annotations

import argparse

from .lattice import SwendsenWang2D


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=8192)
    ap.add_argument("--tile", type=int, nargs=2, default=(16, 8))
    ap.add_argument("--lcg-width", type=int, default=16)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--temperature", type=float, default=2.2691853)
    args = ap.parse_args()
    with SwendsenWang2D(args.L, args.L, tuple(args.tile), args.lcg_width) as sw:
        sw.hot_start(1)
        sw.update(args.temperature, args.sweeps)
        sw.synchronize()
    print(f"ok L={args.L} tile={tuple(args.tile)} sweeps={args.sweeps}")


if __name__ == "__main__":
    main()
