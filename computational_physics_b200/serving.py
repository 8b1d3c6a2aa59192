"""Continuous-batching serving of Swendsen-Wang simulation jobs on one GPU.

A job is (L, T, sweeps, seed): an L x L periodic lattice hot-started from `seed`, swept
`sweeps` times at temperature T with E and M measured every `measure_every` sweeps; its
result is E/N (and |M|/N) averaged over the measurements after the first `discard` fraction,
with a blocking error, plus the exact finite-lattice E/N.

:class:`Server` admits arriving jobs into a :class:`BatchedSW` as slots and HBM budget allow
(first come, first served), keeps their spins, labels and lcg32 streams resident, and sweeps
every admitted job together: a job that arrives while others run joins at the next round.
Each job's sweep budget is counted on the device, so a job stops at exactly its sweep count
and gives the same result as it would alone.  :class:`SequentialServer` is the baseline: jobs
one at a time on the single-lattice path.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import autotune
from ._native import NativeError
from .analysis import binning_error, exact_energy
from .batch import BatchedSW
from .lattice import SwendsenWang2D

__all__ = ["Job", "poisson_jobs", "Server", "SequentialServer", "latency_summary"]


@dataclass
class Job:
    jid: int
    L: int
    T: float
    sweeps: int
    seed: int
    arrival: float = 0.0
    admitted: float | None = None
    done: float | None = None
    result: dict = field(default_factory=dict)

    @property
    def latency(self) -> float | None:
        return None if self.done is None else self.done - self.arrival

    @property
    def site_updates(self) -> int:
        return self.L * self.L * self.sweeps


def poisson_jobs(rate: float, n: int, seed: int = 0, L_range=(32, 2048), T_range=(1.5, 3.5),
                 sweeps_range=(1e3, 1e5)) -> list[Job]:
    """n jobs with Poisson arrivals at `rate` per second; L log-uniform in L_range rounded to a
    multiple of 16, T uniform, sweeps log-uniform, one seed per job."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    L = np.exp(rng.uniform(math.log(L_range[0]), math.log(L_range[1]), size=n))
    L = np.clip(np.round(L / 16) * 16, 16, None).astype(int)
    T = rng.uniform(*T_range, size=n)
    S = np.exp(rng.uniform(math.log(sweeps_range[0]), math.log(sweeps_range[1]), size=n)).astype(int)
    seeds = rng.integers(1, 2 ** 31 - 1, size=n)
    return [Job(i, int(L[i]), float(np.float32(T[i])), int(S[i]), int(seeds[i]), float(t[i])) for i in range(n)]


def _result(samples: np.ndarray, L: int, T: float, discard: float) -> dict:
    n = L * L
    k0 = int(len(samples) * discard)
    E = -samples[k0:, 0].astype(np.float64) / n
    M = np.abs(samples[k0:, 1].astype(np.float64)) / n
    out = {"samples": int(len(samples)), "used": int(len(E)), "exact_E": exact_energy(T, L)}
    if len(E):
        b = binning_error(E, min_blocks=8)
        out.update({"E": b.mean, "E_err": b.error, "absM": float(M.mean()),
                    "z": (b.mean - out["exact_E"]) / b.error if b.error > 0 else float("nan")})
    return out


class Server:
    def __init__(self, hbm_budget_bytes: int, capacity: int = 1024, device: int = 0, measure_every: int = 10,
                 discard: float = 0.1, target_round_ms: float = 2.0, max_rounds: int = 256):
        self.batch = BatchedSW(capacity, hbm_budget_bytes, 16, device)
        self.measure_every = measure_every
        self.discard = discard
        self.target_ms = target_round_ms
        self.max_rounds = max_rounds
        self.table = autotune.load()
        self.rejected: list[Job] = []

    def close(self):
        self.batch.close()

    def _admit(self, job: Job) -> int | None:
        tile, block = autotune.choice(job.L, self.table)
        try:
            lid = self.batch.add(job.L, job.L, job.T, job.seed, tile, block)
        except NativeError as e:
            if e.status == 4:  # SWB_ERR_CAPACITY: no slot or HBM budget left for now
                return None
            raise
        self.batch.hot_start(lid, job.seed)
        self.batch.set_schedule(lid, job.sweeps, self.measure_every)
        return lid

    def run(self, jobs: list[Job], realtime: bool = True) -> list[Job]:
        """Serves `jobs` (arrival times relative to the start).  With realtime=False every job
        is treated as arrived at time 0."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        waiting: deque[Job] = deque()
        running: dict[int, Job] = {}
        round_ms = 1.0
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        while pending or waiting or running:
            now = clock()
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.popleft())
            while waiting:
                lid = self._admit(waiting[0])
                if lid is None:
                    if not running:  # too big for the budget even when the GPU is empty
                        self.rejected.append(waiting.popleft())
                        continue
                    break
                job = waiting.popleft()
                job.admitted = clock()
                running[lid] = job
            if not running:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.01)))
                continue
            k = int(max(1, min(self.max_rounds, self.target_ms / max(round_ms, 1e-3))))
            t_a = time.perf_counter()
            self.batch.sweep(k, measure=True)
            left, _ = self.batch.poll()
            round_ms = 0.7 * round_ms + 0.3 * (time.perf_counter() - t_a) * 1e3 / k
            finished = [lid for lid in running if left[lid] == 0]
            for lid in finished:
                job = running.pop(lid)
                job.result = _result(self.batch.samples(lid), job.L, job.T, self.discard)
                self.batch.remove(lid)
                job.done = clock()
        return jobs


class SequentialServer:
    """Baseline: one job at a time on the single-lattice path, in arrival order."""

    def __init__(self, device: int = 0, measure_every: int = 10, discard: float = 0.1):
        self.device = device
        self.measure_every = measure_every
        self.discard = discard
        self.table = autotune.load()

    def run(self, jobs: list[Job], realtime: bool = True) -> list[Job]:
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        for job in sorted(jobs, key=lambda j: j.arrival):
            if realtime:
                while clock() < job.arrival:
                    time.sleep(min(job.arrival - clock(), 0.01))
            job.admitted = clock()
            tile, _ = autotune.choice(job.L, self.table)
            with SwendsenWang2D(job.L, job.L, tile, 16, job.seed, self.device) as sw:
                sw.hot_start(job.seed)
                sw.update(job.T, job.sweeps, self.measure_every)
                job.result = _result(sw.samples(), job.L, job.T, self.discard)
            job.done = clock()
        return jobs


def latency_summary(jobs: list[Job]) -> dict:
    lat = np.array([j.latency for j in jobs if j.latency is not None])
    if not len(lat):
        return {"jobs": 0}
    span = max(j.done for j in jobs if j.done is not None) - min(j.arrival for j in jobs)
    work = sum(j.site_updates for j in jobs if j.done is not None)
    return {"jobs": int(len(lat)), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": float(span), "site_updates_per_s": work / span}
