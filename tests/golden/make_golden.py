"""Generates the golden fixtures in this directory from the UNMODIFIED reference.

Needs the reference sources (--ref, else $SWB_REFERENCE_DIR, else /root/reference) and the harness built by
``make -C oracle ref``.  Run from the repository root:

    python tests/golden/make_golden.py [--ref /root/reference]

Outputs (all small):
  golden_w16.npz / golden_w8.npz  stage dumps and lcg32 streams from oracle/_ref/libswref{16,8}.so
  exact_ff.json                   printed (K, E/N, C/N) of ising/verification/FF_internalEnergy_specificHeat.c
  ising2d_cli.json                printed results of the reference's own Ising2D program run with
                                  NUM_THREADS equal to the number of tiles (one lcg32 stream per tile)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import RefHarness, num_tiles  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (L0, L1, tx, ty, T, n_sweeps, seed_base); small cases keep full arrays, large ones hashes.
SW_CASES = [
    (16, 16, 16, 8, 2.2691853, 1, 1),
    (32, 16, 16, 8, 2.2691853, 1, 1),
    (64, 64, 16, 8, 2.2691853, 3, 1),
    (64, 64, 8, 8, 2.2691853, 3, 1),
    (128, 128, 16, 8, 2.2691853, 2, 1),   # the CPU config's lattice and tile
    (100, 38, 16, 8, 3.0, 2, 1),          # ragged tiles in both directions
    (18, 10, 16, 8, 2.3, 3, 1),           # one full and one 2-wide tile column
    (32, 32, 32, 4, 2.5, 2, 5),           # tile wider than W, other seed base
    (16, 16, 16, 16, 1.5, 2, 1),          # one tile: both merges wrap onto itself
    (48, 24, 8, 4, 2.0, 4, 3),
    (64, 8, 16, 8, 4.0, 2, 1),            # single tile row
    (2, 2, 16, 8, 2.2691853, 2, 1),       # smallest lattice, tile larger than it
]
HASH_CASES = [
    (256, 256, 16, 8, 2.2691853, 2, 1),
    (1024, 1024, 8, 8, 2.2691853, 2, 1),  # the GPU config's lattice and tile
    (512, 256, 16, 8, 2.0, 3, 1),
]
FULL_LIMIT = 128 * 128


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make(width: int) -> None:
    ref = RefHarness(width)
    assert ref.W == width, (ref.W, width)
    d: dict[str, np.ndarray] = {}
    temps = np.linspace(0.25, 6.0, 512).astype(np.float32)
    temps = np.concatenate([temps, np.float32([2.2691853, 2.2691853142130221, 1.5, 3.5, 2.0, 2.6])])
    d["p_add_T"] = temps
    d["p_add"] = np.array([ref.p_add(float(t)) for t in temps], np.float32)
    d["hot_start_64x32"] = ref.hot_start(64, 32)
    d["hot_start_1024_sha"] = np.frombuffer(bytes.fromhex(sha(ref.hot_start(1024, 1024))), np.uint8)
    seeds = np.arange(1, 33, dtype=np.uint32)
    init = [ref.lcg32_init(int(s)) for s in seeds]
    d["lcg32_seeds"] = seeds
    d["lcg32_state"] = np.stack([x[0] for x in init])
    d["lcg32_a"] = np.stack([x[1] for x in init])
    d["lcg32_c"] = np.stack([x[2] for x in init])
    sizes = np.array([16, 24, 8, 40, 3, 1, 17, 16] * 12, np.uint32)
    d["next_real_sizes"] = sizes
    d["next_real_seed7"] = ref.next_real(7, sizes).view(np.uint32)
    d["next_real_seed1"] = ref.next_real(1, sizes).view(np.uint32)
    cases = []
    for k, (L0, L1, tx, ty, T, ns, sb) in enumerate(SW_CASES + HASH_CASES):
        rng = np.random.default_rng(1000 + k)
        spins = ref.hot_start(L0, L1) if k % 2 == 0 else rng.integers(0, 2, (L1, L0), dtype=np.uint8)
        s_after, bonds, la, lf, rt = ref.run(spins, tx, ty, T, ns, sb)
        key = f"sw{k}"
        cases.append([L0, L1, tx, ty, float(np.float32(T)), ns, sb])
        d[key + "_spins_in"] = spins
        if L0 * L1 <= FULL_LIMIT:
            d[key + "_bonds"] = bonds
            d[key + "_labels_assign"] = la
            d[key + "_labels_final"] = lf
            d[key + "_spins_out"] = s_after
            d[key + "_rng_state"] = rt.state
            d[key + "_rng_a"] = rt.a
            d[key + "_rng_c"] = rt.c
            d[key + "_rng_iteration"] = rt.iteration
        else:
            del d[key + "_spins_in"]
            d[key + "_spins_in_seed"] = np.array([1000 + k, k % 2], np.int64)
            for name, arr in (("bonds", bonds), ("labels_assign", la), ("labels_final", lf),
                              ("spins_out", s_after), ("rng_state", rt.state), ("rng_iteration", rt.iteration)):
                d[key + "_" + name + "_sha"] = np.frombuffer(bytes.fromhex(sha(arr)), np.uint8)
        em = ref.energy_magnetization(s_after)
        d[key + "_em"] = np.array(em, np.float64)
    d["sw_cases"] = np.array(cases, np.float64)
    d["sw_n_full"] = np.array([len(SW_CASES)], np.int64)
    np.savez_compressed(os.path.join(OUT, f"golden_w{width}.npz"), **d)


# (L, num_sweeps, tile_x): small runs, one whose sweep count is not a multiple of the 10-sweep
# measurement block (the loop runs ceil(n/10) blocks and divides by n/10), and the CPU config's
# full protocol (128 x 128, 1000 warm-up + 100000 sweeps, 128 tiles of 16 x 8).
CLI_RUNS = [(32, 200, 16), (64, 100, 16), (32, 205, 16), (128, 100000, 16)]


def make_cli() -> None:
    runs = []
    for (L, sweeps, tile_x) in CLI_RUNS:
        nt = num_tiles(L, L, tile_x, 8)
        env = dict(os.environ, NUM_THREADS=str(nt))
        exe = os.path.join(ROOT, "oracle", "_ref", "Ising2D_w16")
        out = subprocess.run([exe, f"--extent={L}x{L}", f"--num_sweeps={sweeps}"], env=env,
                             capture_output=True, text=True, check=True).stdout
        vals = {}
        for line in out.splitlines():
            if ":" in line and "per spin" in line:
                k, v = line.split(":", 1)
                vals[k.strip()] = v.strip()
        runs.append({"L": L, "num_sweeps": sweeps, "tile": [tile_x, 8], "NUM_THREADS": nt, "printed": vals})
    with open(os.path.join(OUT, "ising2d_cli.json"), "w") as f:
        json.dump(runs, f, indent=1)


def make_exact() -> None:
    """Printed (K, E/N, C/N) of the reference's long-double exact-energy program."""
    exe = os.path.join(ROOT, "oracle", "_ref", "Ising2D_FF_ld")
    rows = []
    for L in (16, 32, 64, 128):
        for K in ("0.44068679350977147", "0.5", "0.44068680351", "0.38461538461538464", "0.3333333333333333"):
            out = subprocess.run([exe, K, str(L), str(L)], capture_output=True, text=True, check=True).stdout.split()
            rows.append({"K": float(K), "L": L, "E": float(out[1]), "C": float(out[2])})
    with open(os.path.join(OUT, "exact_ff.json"), "w") as f:
        json.dump(rows, f, indent=1)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SWB_REFERENCE_DIR", "/root/reference"))
    ap.add_argument("--only", default="", help="comma-separated subset of w16,w8,cli,exact")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}"], check=True)
    only = set(args.only.split(",")) if args.only else {"w16", "w8", "cli", "exact"}
    if "w16" in only:
        make(16)
    if "w8" in only:
        make(8)
    if "cli" in only:
        make_cli()
    if "exact" in only:
        make_exact()


if __name__ == "__main__":
    main()
