"""lcg32 throughput on the GPU, the counterpart of the reference's TestRNG --target program
(random/src/test_rng.cpp): many independent streams, stream i seeded i + 1, each update of a
stream's W lanes yields W numbers in [0, 1).  Prints the last 64 numbers of stream --id, the
time per random number and billions of random numbers per second, as TestRNG does.

    python -m computational_physics_b200.rng_bench [--id=2] [--numbers 16384000000]
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np

from ._native import check, lib


def generate(n_streams: int, updates_per_stream: int, lcg_width: int = 16, seed_base: int = 1,
             report_id: int = 0, device: int = 0) -> dict:
    """One launch: {'report': last 64 numbers of stream report_id, 'checksum': XOR of the bits of
    every number, 'ms': kernel time, 'numbers': numbers generated}."""
    report = np.empty(64, np.float32)
    checksum = ctypes.c_uint32()
    ms = ctypes.c_float()
    check(lib().swb_lcg32_benchmark(n_streams, lcg_width, seed_base, updates_per_stream, report_id,
                                    report.ctypes.data, ctypes.byref(checksum), ctypes.byref(ms), device))
    return {"report": report, "checksum": checksum.value, "ms": ms.value,
            "numbers": n_streams * updates_per_stream * lcg_width}


def benchmark(numbers: int = 16 * 1000 * 1000 * 1024, warmup: int = 1000 * 1024, lcg_width: int = 16,
              n_streams: int = 148 * 512, report_id: int = 0, device: int = 0) -> dict:
    """TestRNG's protocol: a warm-up launch, then one timed launch producing about `numbers`
    numbers (rounded up to whole 64-number buffers per stream).  The default stream count fills
    the 148 SMs of a B200 with 512 streams each."""
    per = 64 // lcg_width

    def updates(n):
        u = -(-n // (n_streams * lcg_width))
        return max(per, -(-u // per) * per)

    generate(n_streams, updates(warmup), lcg_width, 1, report_id, device)
    r = generate(n_streams, updates(numbers), lcg_width, 1, report_id, device)
    r["n_streams"] = n_streams
    r["numbers_per_s"] = r["numbers"] / (r["ms"] * 1e-3)
    return r


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--id", type=int, default=0)
    ap.add_argument("--numbers", type=int, default=16 * 1000 * 1000 * 1024)
    ap.add_argument("--lcg-width", type=int, default=16)
    args = ap.parse_args()
    r = benchmark(args.numbers, lcg_width=args.lcg_width, report_id=args.id)
    print(" ".join(f"{x:g}" for x in r["report"]))
    print(f"Time per random number = {r['ms'] * 1e6 / r['numbers']:g} ns")
    print(f"Billion random numbers per second = {r['numbers_per_s'] / 1e9:g}")


if __name__ == "__main__":
    main()
