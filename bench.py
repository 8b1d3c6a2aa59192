#!/usr/bin/env python
"""Benchmark of the B200 Swendsen-Wang engine; prints ONE JSON line on rank 0.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one Swendsen-Wang sweep over the whole workload.  Workloads (synthetic, seeded):

  batched      512 periodic lattices, side L uniform in {64, 96, 128, 192, 256, 384, 512},
               T uniform in [2.0, 2.6], hot start per lattice seed, one batched sweep per
               step (the headline workload, about 40 M sites)
  plain16384   one 16384^2 lattice at T_c, tile 16x8, lcg32 W = 16, hot start
  plain8192, plain4096   the same at 8192^2 and 4096^2
  plain1024    one 1024^2 lattice at T_c, tile 8x8, lcg32 W = 16, hot start
  serving      Poisson job streams at 10 / 100 / 1000 jobs per second

`value` is spin-updates/s of the whole job with the spins resident in HBM; `e2e` is the same
metric through the C ABI with HOST spin buffers (copies in the timed region).  The reference
arm (--impl reference) times the reference's own CPU path (built from its sources under
oracle/_ref) on this host's cores, on the same workload.

Multi-GPU: one process per GPU (torchrun), no collective on the data path; the time is the
max over ranks.  The batched mix is sharded: every lattice lives on one rank (partition by
device bytes, computational_physics_b200/shard.py), each rank sweeps its share, the value counts
the whole mix (strong scaling), and the per-lattice observables are gathered on rank 0.  Serving
shards the job stream the same way.  A single lattice does not shard (cross-GPU labelling would
need iterative label exchange): plain workloads run one replica per rank (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

T_C = 2.2691853
MIX_SIDES = (64, 96, 128, 192, 256, 384, 512)
MIX_COUNT = 512
MIX_SEED = 20260
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


# ---------------------------------------------------------------------------------------------
# workloads

def mix_workload(count: int = MIX_COUNT, seed: int = MIX_SEED):
    rng = np.random.default_rng(seed)
    sides = rng.choice(MIX_SIDES, size=count)
    temps = rng.uniform(2.0, 2.6, size=count).astype(np.float32)
    seeds = rng.integers(1, 2 ** 31 - 1, size=count)
    return [(int(L), float(T), int(s)) for L, T, s in zip(sides, temps, seeds)]


PLAIN = {
    "plain16384": dict(L=16384, tile=(16, 8), W=16, T=T_C),
    "plain8192": dict(L=8192, tile=(16, 8), W=16, T=T_C),
    "plain4096": dict(L=4096, tile=(16, 8), W=16, T=T_C),
    "plain1024": dict(L=1024, tile=(8, 8), W=16, T=T_C),
}


# ---------------------------------------------------------------------------------------------
# distributed plumbing (control plane only: barrier and max-reduce of device times)

class Dist:
    """One process per GPU: NCCL on a GPU box (gloo where there is no GPU, as in the CPU tests).
    Only a barrier and a max-reduce of the device-measured times go over it."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = "gloo"
            if torch.cuda.is_available():
                backend = "nccl"
                torch.cuda.set_device(self.local_rank)
                self.device = torch.device("cuda", self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.device is not None:
                self.pg.barrier(device_ids=[self.local_rank])
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def gather_object(self, obj):
        """Every rank's `obj` as a list on rank 0 (None on the other ranks); host data only."""
        if not self.pg:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self.pg.gather_object(obj, out, dst=0)
        return out

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled every 10 ms by NVML (read-only
    queries) from a thread while the timed region runs, plus one sample as it ends, so that even
    a region of a few milliseconds has samples.  Falls back to nvidia-smi (every 200 ms) when
    NVML is unavailable."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, device: int, period_s: float = 0.01):
        self.device = device
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.handle = None
        self.stop = threading.Event()
        self.lines: list[str] = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        self.nvml = pynvml
        try:  # the CUDA device by UUID (NVML numbers every GPU of the host, CUDA only the visible ones)
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _nvml_sample(self):
        n, h = self.nvml, self.handle
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)
        get = getattr(n, "nvmlDeviceGetCurrentClocksEventReasons", None) or n.nvmlDeviceGetCurrentClocksThrottleReasons
        r = get(h)
        flags = ["Active" if r & bit else "Not Active" for bit in self.REASONS.values()]
        self.lines.append(",".join([str(self.device), str(sm), str(mx), "", hex(r), *flags]))

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            self.handle = self._nvml_handle()
            self._nvml_sample()
            self.lines.clear()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:   # first sample before timing starts
                time.sleep(0.02)
            self.lines.clear()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml is not None:
            try:
                self._nvml_sample()  # the end of the timed region
            except Exception:
                pass
            self.stop.set()
            self.thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def hbm_peak() -> tuple[float, str]:
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------------------------
# algorithmic bytes (roofline numerators), per site or per tile

def assign_bytes(n_sites: int, n_tiles: int, W: int) -> float:
    """k_assign: spins read (1 B/site) + block-local labels written (4 B/site) + the tile's
    lcg32 streams read and written (W state words + W parameter bytes + 1 counter)."""
    return n_sites * 5 + n_tiles * 2 * (W * 5 + 4)


# DRAM traffic of one assign pass over a workload (dram__bytes_read.sum + dram__bytes_write.sum)
# from one ncu capture of the same kernel, per site: the batched mix of 512 lattices (39,603,200
# sites; the round runs its two lattice groups as two launches: 33,125,632 + 33,147,904 B read,
# 36,334,848 + 35,846,400 B written) and one 8192 x 8192 lattice, tile 16 x 8 (111,228,928 B read
# + 253,859,584 B written).  Traffic grows with the sites swept, so other sizes scale by their
# site count.
ASSIGN_TRAFFIC_PER_SITE = {"kb_assign": (33_125_632 + 33_147_904 + 36_334_848 + 35_846_400) / 39_603_200,
                           "k_assign": (111_228_928 + 253_859_584) / 8192 ** 2}


def flip_bytes(n_sites: int) -> float:
    """k_flip: labels read (4 B/site) + spins read and written (2 B/site)."""
    return n_sites * 6


# ---------------------------------------------------------------------------------------------
# reference arm and CPU baseline: the reference's own CPU path in a child process

def _ref_width() -> int:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        flags = ""
    return 16 if " avx512f" in flags else 8


def ref_worker(args) -> None:
    """Child process: times SwendsenWang_2D<LCG32, CPU>::Update of the reference."""
    from oracle import RefHarness, have_ref
    spec = json.loads(args.ref_spec)
    width = _ref_width()
    if not have_ref(width):
        print(json.dumps({"error": f"oracle/_ref/libswref{width}.so is missing"}))
        return
    ref = RefHarness(width)
    sides = spec["sides"]
    temps = spec["temps"]
    spins = [ref.hot_start(L, L) for L in sides]
    threads = spec["threads"]
    ref.cpu_sweep_many(sides, temps, spins, spec["warmup"], threads)
    secs = ref.cpu_sweep_many(sides, temps, spins, spec["sweeps"], threads)
    sites = sum(L * L for L in sides)
    print(json.dumps({"seconds": secs, "site_updates": sites * spec["sweeps"], "threads": threads, "W": width}))


def run_ref_child(sides, temps, sweeps: int, warmup: int, threads: int) -> dict:
    spec = json.dumps({"sides": list(map(int, sides)), "temps": list(map(float, temps)), "sweeps": sweeps,
                       "warmup": warmup, "threads": threads})
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--_ref-worker", "--ref-spec", spec],
                         capture_output=True, text=True, timeout=900)
    for line in reversed(out.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    return {"error": (out.stderr or out.stdout)[-300:]}


def reference_sample(workload: str, budget_s: float = 20.0):
    """The bounded sample of the workload the CPU runs: (sides, temps, description)."""
    if workload == "batched":
        mix = mix_workload()
        sides = [L for L, _, _ in mix]
        temps = [T for _, T, _ in mix]
        return sides, temps, f"the full {len(mix)}-lattice mix"
    p = PLAIN[workload]
    return [p["L"]], [p["T"]], f"one {p['L']}^2 lattice at T={p['T']}"


def cpu_baseline(workload: str) -> dict:
    threads = os.cpu_count() or 1
    sides, temps, desc = reference_sample(workload)
    probe = run_ref_child(sides, temps, 1, 1, threads)
    if "error" in probe:
        return {"value": None, "unit": "spin-updates/s", "cores": threads, "kind": "reference",
                "sample": desc, "error": probe["error"]}
    per_sweep = max(probe["seconds"], 1e-6)
    sweeps = max(1, min(50, int(15.0 / per_sweep)))
    r = run_ref_child(sides, temps, sweeps, 1, threads)
    if "error" in r:
        return {"value": None, "unit": "spin-updates/s", "cores": threads, "kind": "reference",
                "sample": desc, "error": r["error"]}
    return {"value": r["site_updates"] / r["seconds"], "unit": "spin-updates/s", "cores": threads,
            "kind": "reference",
            "sample": f"{sweeps} sweeps of {desc} after 1 warmup sweep, reference CPU path "
                      f"(SwendsenWang_2D<LCG32, CPU>::Update, W={r['W']}, NUM_THREADS={threads})",
            "seconds": r["seconds"]}


def run_reference_arm(args, dist: Dist) -> None:
    if dist.rank != 0:
        return
    threads = os.cpu_count() or 1
    sides, temps, desc = reference_sample(args.workload)
    probe = run_ref_child(sides, temps, 1, 1, threads)
    metric, unit = "SW spin-updates/s", "spin-updates/s"
    if "error" in probe:
        print(json.dumps({"impl": "reference", "unavailable": probe["error"]}))
        return
    per_sweep = max(probe["seconds"], 1e-6)
    steps = args.steps
    while steps > 1 and per_sweep * (steps + args.warmup) > 150:
        steps -= 1
    r = run_ref_child(sides, temps, steps, args.warmup, threads)
    if "error" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["error"]}))
        return
    value = r["site_updates"] / r["seconds"]
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic", "config": workload_config(args.workload),
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "reference",
                         "sample": f"{steps} sweeps of {desc}, reference CPU path, W={r['W']}"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def workload_config(name: str) -> dict:
    if name == "batched":
        mix = mix_workload()
        return {"workload": "batched SW, 512 periodic lattices, L uniform in {64,96,128,192,256,384,512}, "
                            "T uniform in [2.0, 2.6], hot start, one sweep of every lattice per step",
                "lattices": len(mix), "sites": sum(L * L for L, _, _ in mix), "tile": "autotuned per L",
                "lcg_width": 16, "l2": "inputs larger than L2"}
    p = PLAIN[name]
    big = p["L"] * p["L"] * 5 > 126e6
    return {"workload": f"plain SW, one periodic {p['L']}x{p['L']} lattice, T={p['T']}, hot start",
            "tile": list(p["tile"]), "lcg_width": p["W"], "sites": p["L"] * p["L"],
            "l2": "inputs larger than L2" if big else "L2 flushed between timed sweeps"}


# ---------------------------------------------------------------------------------------------
# our arm

def bench_plain(args, dist: Dist, cp) -> dict:
    p = PLAIN[args.workload]
    L, tile, W, T = p["L"], p["tile"], p["W"], p["T"]
    n = L * L
    sw = cp.SwendsenWang2D(L, L, tile, W, seed_base=1, device=dist.local_rank)
    sw.hot_start(1)
    sw.update(T, args.warmup)
    sw.synchronize()
    big = n * 5 > 126e6
    flush = None
    if not big:
        flush = cp.SwendsenWang2D(4096, 4096, (16, 8), 16, device=dist.local_rank)  # 16 MB spins + 64 MB labels
    launches0 = cp.kernel_launches()
    dist.barrier()
    with ClockSampler(dist.local_rank) as clocks:
        if big:
            ms = float(sw.sweep_timed(T, args.steps)[0])
        else:
            ms = 0.0
            for _ in range(args.steps):
                flush.cold_start(0)
                flush.cold_start(1)
                flush.synchronize()
                ms += float(sw.sweep_timed(T, 1)[0])
    launches = cp.kernel_launches() - launches0 - (0 if big else 2 * args.steps)
    if flush is not None:
        flush.close()
    dist.barrier()
    ms_max = dist.max(ms)
    value = dist.world * n * args.steps / (ms_max / 1e3)
    # per-kernel times for the roofline (separate instrumented pass)
    k = sw.sweep_timed(T, max(3, min(args.steps, 20)), per_kernel=True)
    nk = max(3, min(args.steps, 20))
    n_tiles, _ = sw.rng_shape()
    peak, peak_kind = hbm_peak()
    a_ms = float(k[1]) / nk
    ab = assign_bytes(n, n_tiles, W)
    fb = flip_bytes(n)
    # e2e through host buffers
    spins_in = cp.lattice.pinned_empty((L, L), np.uint8)
    spins_out = cp.lattice.pinned_empty((L, L), np.uint8)
    spins_in[:] = sw.get_spins()
    em = np.zeros(2)
    import time as _t
    sw.update_host(T, spins_in, spins_out, em)
    e2e_steps = max(3, min(args.steps, 10))
    dist.barrier()
    t0 = _t.perf_counter()
    for _ in range(e2e_steps):
        sw.update_host(T, spins_in, spins_out, em)
        spins_in, spins_out = spins_out, spins_in
    e2e_s = dist.max(_t.perf_counter() - t0)
    e2e = dist.world * n * e2e_steps / e2e_s
    sw.close()
    return {
        "value": value, "ms_per_step": ms_max / args.steps, "launches": launches, "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "kernel": "k_assign", "achieved": ab / (a_ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": ab / (a_ms / 1e3) / 1e9 / peak,
                     "traffic": ASSIGN_TRAFFIC_PER_SITE["k_assign"] * n, "peak_kind": peak_kind,
                     "bytes_per_launch": ab, "ms_per_launch": a_ms},
        "kernels_ms_per_sweep": {"assign": a_ms, "merge": float(k[2]) / nk, "resolve_flip": float(k[3]) / nk},
        "flip_GBs": fb / (float(k[3]) / nk / 1e3) / 1e9,
        "e2e": {"value": e2e, "unit": "spin-updates/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": n + 16},
    }


def mix_shards(world: int, lcg_width: int = 16):
    """The mix's lattice indices per rank, balanced by the batched engine's device bytes."""
    from computational_physics_b200 import autotune, shard
    table = autotune.load(lcg_width=lcg_width)
    weights = [shard.lattice_bytes(L, L, autotune.choice(L, table)[0], lcg_width) for L, _, _ in mix_workload()]
    parts = shard.partition(weights, world)
    return parts, shard.imbalance(parts, weights)


def mix_observables(b, ids, index) -> dict:
    """{mix index: [e, m]} of the lattices' current spins (integer sums over sites of
    s (s_right + s_down) and s), read back to the host."""
    out = {}
    for lid, k in zip(ids, index):
        s = b.get_spins(lid).astype(np.int64) * 2 - 1
        e = int(np.sum(s * (np.roll(s, -1, axis=1) + np.roll(s, -1, axis=0))))
        out[k] = [e, int(s.sum())]
    return out


def build_mix(cp, device: int, lcg_width: int = 16, subset=None):
    """The batched engine holding the mix's lattices (all, or the indices in `subset`)."""
    from computational_physics_b200 import autotune
    table = autotune.load(lcg_width=lcg_width)
    mix = mix_workload()
    if subset is not None:
        mix = [mix[k] for k in subset]
    b = cp.BatchedSW(capacity=max(1, len(mix)), lcg_width=lcg_width, device=device)
    ids, tiles = [], []
    for L, T, seed in mix:
        tile, block = autotune.choice(L, table)
        lid = b.add(L, L, T, seed, tile, block)
        b.hot_start(lid, seed)
        ids.append(lid)
        tiles.append((tile, block))
    return b, mix, ids, tiles, table


def plain_loop(cp, mix, tiles, steps: int, device: int) -> dict:
    """The same mix swept by looping the single-lattice path (three or four launches per
    lattice per sweep, each lattice on its own stream)."""
    handles = []
    for (L, T, seed), (tile, _) in zip(mix, tiles):
        h = cp.SwendsenWang2D(L, L, tile, 16, seed_base=seed, device=device)
        h.hot_start(seed)
        handles.append((h, T))
    for h, T in handles:
        h.update(T, 2)
    for h, _ in handles:
        h.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for h, T in handles:
            h.update(T, 1)
    for h, _ in handles:
        h.synchronize()
    secs = time.perf_counter() - t0
    sites = sum(L * L for L, _, _ in mix)
    for h, _ in handles:
        h.close()
    return {"value": sites * steps / secs, "unit": "spin-updates/s", "steps": steps,
            "timing": "host wall clock around the loop, all streams synchronized"}


def energy_gate(cp, device: int, warmup: int = 1000, sweeps: int = 10000, every: int = 10) -> dict:
    """Every lattice of the mix: 1000 warmup + 10000 sweeps measured every 10, E/N against the
    exact finite-lattice value with a binned (autocorrelation-aware) error."""
    from computational_physics_b200.analysis import gate_energy
    b, mix, ids, tiles, _ = build_mix(cp, device)
    b.sweep(warmup)
    for lid in ids:
        b.set_schedule(lid, sweeps, every)
    t0 = time.perf_counter()
    b.sweep(sweeps, measure=True)
    b.synchronize()
    secs = time.perf_counter() - t0
    z = []
    worst = None
    for lid, (L, T, _) in zip(ids, mix):
        g = gate_energy(b.samples(lid), L, L, T)
        z.append(g["z"])
        if worst is None or abs(g["z"]) > abs(worst["z"]):
            worst = {"L": L, "T": T, **g}
    b.close()
    z = np.array(z)
    return {"lattices": len(z), "within_2sigma": int(np.sum(np.abs(z) <= 2)), "frac_within_2sigma":
            float(np.mean(np.abs(z) <= 2)), "max_abs_z": float(np.max(np.abs(z))), "mean_z": float(np.mean(z)),
            "chi2_per_dof": float(np.mean(z * z)), "worst": worst, "seconds": secs,
            "protocol": f"{warmup} warmup + {sweeps} sweeps, measured every {every}, blocking error"}


def bench_batched(args, dist: Dist, cp) -> dict:
    """The 512-lattice mix, sharded: each lattice lives on one rank (partition by device bytes),
    every rank sweeps its share, and the value counts the whole mix over the slowest rank."""
    from computational_physics_b200 import shard
    dev = dist.local_rank
    parts, imbalance = mix_shards(dist.world)
    mine = parts[dist.rank]
    b, mix, ids, tiles, table = build_mix(cp, dev, subset=mine)
    sites = sum(L * L for L, _, _ in mix)                      # this rank's share
    sites_all = sum(L * L for L, _, _ in mix_workload())       # the whole mix
    b.sweep(args.warmup)
    b.synchronize()
    launches0 = cp.kernel_launches()
    dist.barrier()
    with ClockSampler(dev) as clocks:
        ms = float(b.sweep_timed(args.steps)[0])
    launches = cp.kernel_launches() - launches0
    dist.barrier()
    ms_max = dist.max(ms)
    value = sites_all * args.steps / (ms_max / 1e3)
    nk = max(3, min(args.steps, 20))
    k = b.sweep_timed(nk, per_kernel=True)
    a_ms = float(k[1]) / nk
    n_tiles = 0
    for lid in ids:
        n_tiles += b.info(lid)["tiles"]
    ab = assign_bytes(sites, n_tiles, 16)
    peak, peak_kind = hbm_peak()
    # e2e: every step copies all spins in from pinned host memory and back out; the lattices'
    # host buffers are consecutive slices of one pinned arena per direction (BatchedSW.host_io).
    # The steps run as one pipelined call (update_host_io_rounds: a lattice group's next copy in
    # starts once its copy out has landed); one call per step is timed beside it.
    io = b.host_io(ids)
    for lid, x in zip(ids, io.inputs):
        x[:] = b.get_spins(lid)
    b.update_host_io(io)
    io.swap()
    b.update_host_io_rounds(io, 2)
    e2e_steps = max(3, min(args.steps, 20))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        b.update_host_io(io)
        io.swap()
    e2e_sync_s = dist.max(time.perf_counter() - t0)
    dist.barrier()
    t0 = time.perf_counter()
    b.update_host_io_rounds(io, e2e_steps)
    e2e_s = dist.max(time.perf_counter() - t0)
    # per-lattice observables of the final state, gathered on rank 0 (control plane only)
    merged = shard.gather_results(mix_observables(b, ids, mine), dist.gather_object)
    b.close()
    res = {
        "value": value, "ms_per_step": ms_max / args.steps, "launches": launches, "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "kernel": "kb_assign", "achieved": ab / (a_ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": ab / (a_ms / 1e3) / 1e9 / peak,
                     "traffic": ASSIGN_TRAFFIC_PER_SITE["kb_assign"] * sites, "peak_kind": peak_kind,
                     "bytes_per_launch": ab, "ms_per_launch": a_ms},
        "kernels_ms_per_sweep": {"assign": a_ms, "merge": float(k[2]) / nk, "resolve_flip": float(k[3]) / nk},
        "e2e": {"value": sites_all * e2e_steps / e2e_s, "unit": "spin-updates/s",
                "h2d_bytes_per_step": sites_all, "d2h_bytes_per_step": sites_all,
                "api": "swb_batch_update_host_rounds: the steps as one pipelined call through two pinned host arenas",
                "one_step_per_call": sites_all * e2e_steps / e2e_sync_s},
        "tiles": {str(L): [list(t), list(bl)] for (L, _, _), (t, bl) in sorted(zip(mix, tiles))},
        "autotune_table": table.get("device", "none"),
    }
    if merged is not None:
        n_all = [L * L for L, _, _ in mix_workload()]
        res["shard"] = {"ranks": dist.world, "lattices_per_rank": [len(p) for p in parts],
                        "bytes_imbalance": imbalance, "lattices_gathered": len(merged),
                        "mean_E_per_site": float(np.mean([-merged[k][0] / n_all[k] for k in merged]))}
    if dist.world == 1 and not args.quick:
        pl = plain_loop(cp, mix, tiles, max(3, min(args.steps, 10)), dev)
        res["plain_loop"] = pl
        res["batched_vs_plain_loop"] = value / pl["value"]
        res["energy_gate"] = energy_gate(cp, dev)
    return res


def plain_subrecord(cp, dev: int, name: str = "plain16384", sweeps: int = 100) -> dict:
    """One single-lattice workload beside the headline: ms per sweep, per-kernel ms and the
    fraction of the HBM roofline by the algorithmic bytes per sweep (17.1 B/site at 16 x 8)."""
    p = PLAIN[name]
    L, tile, W, T = p["L"], p["tile"], p["W"], p["T"]
    n = L * L
    with cp.SwendsenWang2D(L, L, tile, W, seed_base=1, device=dev) as sw:
        sw.hot_start(1)
        sw.update(T, 5)
        sw.synchronize()
        ms = float(sw.sweep_timed(T, sweeps)[0]) / sweeps
        k = sw.sweep_timed(T, 20, per_kernel=True) / 20
        n_tiles, _ = sw.rng_shape()
    peak, peak_kind = hbm_peak()
    # algorithmic bytes per sweep: 11 B per site (spins and labels) plus every tile's lcg32 state
    # (3 W + 1 words) read and written in each of the two phases that draw
    sweep_bytes = n * 11 + n_tiles * 4 * (12 * W + 4)
    return {"workload": name, "sites": n, "ms_per_sweep": ms, "value": n / (ms / 1e3),
            "kernels_ms": {"assign": float(k[1]), "merge": float(k[2]), "resolve_flip": float(k[3])},
            "bytes_per_sweep": sweep_bytes, "hbm_frac": sweep_bytes / (ms / 1e3) / 1e9 / peak, "peak": peak,
            "peak_kind": peak_kind}


SERVING_RATES = (10.0, 100.0, 1000.0)
SERVING_JOBS = 200            # jobs per rate
SERVING_BASELINE_JOBS = 40    # the first jobs of the stream, one at a time on the single-lattice path
SERVING_SEED = 20260


def serving_run(dist: Dist, n_jobs: int = SERVING_JOBS, baseline_jobs: int = SERVING_BASELINE_JOBS) -> dict:
    """Continuous-batching serving of one job set (L log-uniform in [32, 2048] rounded to 16, T
    uniform in [1.5, 3.5], sweeps log-uniform in [1e3, 1e5], a seed per job) arriving as a
    Poisson stream at 10, 100 and 1000 jobs per second, under a 32 GB HBM budget per GPU.
    Sharded: every job is served by one rank (partition by site updates); job records are
    gathered on rank 0, which gets the summary (other ranks: None).  The baseline serves the
    first `baseline_jobs` jobs one at a time on the single-lattice path, back to back."""
    from computational_physics_b200 import serving, shard
    per_rate = {}
    work = span = 0.0
    for rate in SERVING_RATES:
        jobs = serving.poisson_jobs(rate, n_jobs, seed=SERVING_SEED)
        mine = shard.shard_of([j.site_updates for j in jobs], dist.world, dist.rank)
        local = [jobs[k] for k in mine]
        srv = serving.Server(32 << 30, device=dist.local_rank)
        try:
            srv.run(local, realtime=True)
        finally:
            srv.close()
        recs = {j.jid: [j.arrival, j.admitted, j.done, j.site_updates, j.result.get("z")] for j in local}
        merged = shard.gather_results(recs, dist.gather_object)
        rejected = dist.gather_object(len(srv.rejected))
        bypassed = dist.gather_object(srv.bypassed)
        if merged is None:
            continue
        for j in jobs:
            j.arrival, j.admitted, j.done = merged[j.jid][0], merged[j.jid][1], merged[j.jid][2]
        summ = serving.latency_summary(jobs)
        zs = np.array([merged[k][4] for k in merged if merged[k][4] is not None and np.isfinite(merged[k][4])])
        summ.update(rejected=int(sum(rejected)), bypassed=int(sum(bypassed)),
                    jobs_within_2sigma=float(np.mean(np.abs(zs) <= 2)) if len(zs) else None)
        per_rate[str(int(rate))] = summ
        work += sum(j.site_updates for j in jobs if j.done is not None)
        span += summ.get("makespan_s", 0.0)
    base = None
    if dist.rank == 0:
        base_jobs = serving.poisson_jobs(SERVING_RATES[0], n_jobs, seed=SERVING_SEED)[:baseline_jobs]
        t0 = time.perf_counter()
        serving.SequentialServer(device=dist.local_rank).run(base_jobs, realtime=False)
        secs = time.perf_counter() - t0
        base = {"jobs": len(base_jobs), "site_updates_per_s": sum(j.site_updates for j in base_jobs) / secs,
                "seconds": secs, "timing": "the first jobs of the same stream, back to back, host wall clock"}
    if dist.rank != 0:
        return None
    return {"per_rate": per_rate, "value": work / span if span else 0.0, "sequential_baseline": base,
            "jobs_per_rate": n_jobs, "ranks": dist.world}


def bench_serving(args, dist: Dist, cp) -> None:
    """The serving workload on its own (serving_run); prints its own JSON line (rank 0)."""
    with ClockSampler(dist.local_rank) as clocks:
        r = serving_run(dist)
    if dist.rank != 0:
        return
    n = r["jobs_per_rate"]
    span = sum(v.get("makespan_s", 0.0) for v in r["per_rate"].values())
    print(json.dumps({
        "metric": "SW spin-updates/s", "value": r["value"], "unit": "spin-updates/s", "n_gpus": dist.world,
        "steps": n, "warmup": 0, "ms_per_step": 1e3 * span / (len(SERVING_RATES) * n), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "serving: Poisson arrivals at 10/100/1000 per s, L log-uniform [32, 2048], "
                               "T uniform [1.5, 3.5], sweeps log-uniform [1e3, 1e5], 32 GB HBM budget per GPU",
                   "jobs_per_rate": n, "parallelism": f"job shards x{dist.world}"},
        "serving": r["per_rate"], "sequential_baseline": r["sequential_baseline"], "clocks": clocks.summary(),
    }))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", *PLAIN, "serving"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip the plain-loop comparison and the energy gate")
    ap.add_argument("--_ref-worker", dest="ref_worker_mode", action="store_true")
    ap.add_argument("--ref-spec", default="")
    args = ap.parse_args()
    if args.ref_worker_mode:
        ref_worker(args)
        return
    args.warmup = max(args.warmup, 3)
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference_arm(args, dist)
            return
        import computational_physics_b200 as cp
        if cp.device_count() < 1:
            raise RuntimeError("no CUDA device")
        if args.workload == "serving":
            bench_serving(args, dist, cp)
            return
        r = bench_batched(args, dist, cp) if args.workload == "batched" else bench_plain(args, dist, cp)
        if dist.rank != 0:
            return
        line = {
            "metric": "SW spin-updates/s", "value": r["value"], "unit": "spin-updates/s", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "strong" if args.workload == "batched" else "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {**workload_config(args.workload),
                       "parallelism": (f"lattice shards x{dist.world}" if args.workload == "batched"
                                       else f"replicas x{dist.world}")},
            "roofline": r["roofline"], "e2e": r["e2e"], "gpu_launches": r["launches"], "clocks": r["clocks"],
            "kernels_ms_per_sweep": r["kernels_ms_per_sweep"],
        }
        for key in ("plain_loop", "batched_vs_plain_loop", "energy_gate", "tiles", "autotune_table", "shard"):
            if key in r:
                line[key] = r[key]
        if args.workload == "batched" and dist.world == 1 and not args.quick:
            line["plain16384"] = plain_subrecord(cp, dist.local_rank)
            sv = serving_run(dist)
            line["serving"] = {"value": sv["value"], "unit": "spin-updates/s", "per_rate": sv["per_rate"],
                               "sequential_baseline": sv["sequential_baseline"], "jobs_per_rate": sv["jobs_per_rate"]}
        if dist.world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload)
        print(json.dumps(line))
    finally:
        dist.close()


if __name__ == "__main__":
    main()
