"""Generates c3_sha.json: SHA-256 digests of one recorded sweep at the bandwidth-scaling sizes.

Workload per size L in {4096, 8192, 16384}: periodic L x L lattice, hot start (srand48(1), the
reference's Lattice<2> constructor), tile 16 x 8, lcg32 width 16, one stream per tile seeded
1 + tile id, T = 2.2691853; two sweeps, then the recorded third sweep.  Digests (of the raw
row-major arrays) of the third sweep's bonds, final labels, flipped spins and lcg32 streams come
from the CPU restatement (oracle/sw_oracle.c).  The labels of the bonds inside each 128 x 32
block (the GPU path's assign-phase output) are recorded too, with the block shape they assume.

When the reference harness (oracle/_ref/libswref16.so, built by ``make -C oracle ref``) is
present, the 4096 x 4096 case is also run through the unmodified reference sources and must
agree digest for digest; the file records whether that check ran.

Run from the repository root (needs about 6 GB of host memory and a few minutes):

    python tests/golden/make_c3_fixtures.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import Oracle, RefHarness, have_ref, num_tiles  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c3_sha.json")
SIZES = (4096, 8192, 16384)
TILE = (16, 8)
BLOCK = (128, 32)
W = 16
T = 2.2691853
SWEEPS_BEFORE = 2


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def oracle_case(o: Oracle, L: int) -> dict:
    spins = o.hot_start(L, L, 1)
    rng = o.rng_init(W, num_tiles(L, L, *TILE), 1)
    for _ in range(SWEEPS_BEFORE):
        o.sweep(spins, TILE[0], TILE[1], rng, T=T)
    spins_in = sha(spins)
    bonds, _, lf = o.sweep(spins, TILE[0], TILE[1], rng, T=T, dumps=True)
    lb = o.block_labels(bonds, *BLOCK)
    return {"spins_in": spins_in, "bonds": sha(bonds), "labels_block": sha(lb), "labels_final": sha(lf),
            "spins_out": sha(spins), "rng_state": sha(rng.state), "rng_iteration": sha(rng.iteration)}


def reference_case(L: int) -> dict:
    ref = RefHarness(W)
    spins = ref.hot_start(L, L)
    s, bonds, _, lf, r = ref.run(spins, TILE[0], TILE[1], T, n_sweeps=SWEEPS_BEFORE + 1, seed_base=1)
    return {"bonds": sha(bonds), "labels_final": sha(lf), "spins_out": sha(s), "rng_state": sha(r.state),
            "rng_iteration": sha(r.iteration)}


def main() -> None:
    o = Oracle()
    cases = {}
    for L in SIZES:
        t0 = time.time()
        cases[str(L)] = oracle_case(o, L)
        print(f"L={L}: {time.time() - t0:.1f} s", flush=True)
    cross = False
    if have_ref(W):
        r = reference_case(SIZES[0])
        for k, v in r.items():
            if cases[str(SIZES[0])][k] != v:
                raise SystemExit(f"restatement and reference differ at L={SIZES[0]} in {k}")
        cross = True
        print(f"L={SIZES[0]}: reference harness agrees", flush=True)
    doc = {"tile": list(TILE), "block": list(BLOCK), "lcg_width": W, "temperature": T, "seed_base": 1,
           "hot_start_seed": 1, "sweeps_before": SWEEPS_BEFORE, "reference_cross_checked": [SIZES[0]] if cross else [],
           "cases": cases}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
