"""Continuous-batching serving of Swendsen-Wang simulation jobs on one GPU.

A job is (L, T, sweeps, seed): an L x L periodic lattice hot-started from `seed`, swept
`sweeps` times at temperature T with E and M measured every `measure_every` sweeps; its
result is E/N (and |M|/N) averaged over the measurements after the first `discard` fraction,
with a blocking error, plus the exact finite-lattice E/N, and the raw (e, m) series.

:class:`Server` admits arriving jobs into a :class:`BatchedSW` as slots and HBM budget allow,
keeps their spins, labels and lcg32 streams resident, and sweeps every admitted job together:
a job that arrives while others run joins at the next round.  Each job's sweep budget is
counted on the device, so a job stops at exactly its sweep count and gives the same result as
it would alone.  The host loop never waits on the device to learn progress: every round
sweeps every unfinished job once, so the host knows in which submitted round each job
finishes, marks that point on the stream (swb_batch_mark) and learns its device completion
time without blocking (swb_batch_mark_query); it keeps the next rounds queued meanwhile.
Admission is first come, first served with a bounded bypass: when the head of the queue does
not fit, up to `bypass_window` smaller waiting jobs behind it may go first, at most
`max_bypass` times per head job.  :class:`SequentialServer` is the baseline: jobs one at a time
on the single-lattice path.
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
    multiple of 16, T uniform, sweeps log-uniform, one seed per job.  The same seed gives the
    same jobs at every rate (only the arrival times scale with 1 / rate)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0, size=n)) / rate
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
    out = {"samples": int(len(samples)), "used": int(len(E)), "exact_E": exact_energy(T, L), "series": samples}
    if len(E):
        b = binning_error(E, min_blocks=8)
        out.update({"E": b.mean, "E_err": b.error, "absM": float(M.mean()),
                    "z": (b.mean - out["exact_E"]) / b.error if b.error > 0 else float("nan")})
    return out


class Server:
    def __init__(self, hbm_budget_bytes: int, capacity: int = 1024, device: int = 0, measure_every: int = 10,
                 discard: float = 0.1, target_round_ms: float = 4.0, max_rounds: int = 512, bypass_window: int = 16,
                 max_bypass: int = 64, max_in_flight: int = 2):
        self.batch = BatchedSW(capacity, hbm_budget_bytes, 16, device)
        self.measure_every = measure_every
        self.discard = discard
        self.target_ms = target_round_ms
        self.max_rounds = max_rounds
        self.bypass_window = bypass_window
        self.max_bypass = max_bypass
        self.max_in_flight = max_in_flight
        self.table = autotune.load()
        self.rejected: list[Job] = []
        self.bypassed = 0   # admissions that went ahead of a waiting head job

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
        b = self.batch
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        waiting: list[Job] = []
        running: dict[int, Job] = {}      # slot -> job still sweeping (host count of its rounds left)
        left: dict[int, int] = {}         # slot -> rounds still to submit for its job
        finishing: dict[int, list[int]] = {}  # mark -> slots whose last sweep precedes it
        finished: list[int] = []          # slots done and read, memory not yet released
        in_flight: deque[tuple[int, int]] = deque()  # (mark, rounds) submitted, not yet passed
        head_skips = 0
        rate = 1.0                        # rounds per ms, measured
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        origin_mark = b.mark()            # device time origin ~ host time t_origin
        t_origin = clock()
        b.mark_done(origin_mark)
        last_mark_time = (0.0, 0)          # (device s, rounds) of the last passed mark

        def release_finished():
            while finished:
                b.remove(finished.pop())

        while pending or waiting or running or in_flight:
            now = clock()
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.popleft())
            # admission: the head first; up to bypass_window jobs behind it may go ahead when
            # it does not fit, at most max_bypass times for one head
            i = 0
            while i < len(waiting) and i <= self.bypass_window:
                if i > 0 and head_skips >= self.max_bypass:
                    break
                lid = self._admit(waiting[i])
                if lid is None and finished:
                    release_finished()
                    lid = self._admit(waiting[i])
                if lid is None:
                    if i == 0 and not running and not in_flight:
                        self.rejected.append(waiting.pop(0))  # too big even for an empty GPU
                        continue
                    i += 1
                    continue
                job = waiting.pop(i)
                if i > 0:
                    head_skips += 1
                    self.bypassed += 1
                else:
                    head_skips = 0
                job.admitted = clock()
                running[lid] = job
                left[lid] = job.sweeps
            # keep up to max_in_flight submissions queued: rounds until the next job finishes,
            # fewer when an arrival is due sooner
            if running and len(in_flight) < self.max_in_flight and any(left[l] for l in running):
                r = min(left[l] for l in running if left[l])
                cap = self.max_rounds
                if pending and realtime:
                    cap = max(1, int(rate * 1e3 * max(pending[0].arrival - now, 0.0)))
                r = int(max(1, min(r, cap, max(1, rate * self.target_ms))))
                b.sweep(r, measure=True)
                m = b.mark()
                in_flight.append((m, r))
                for l in running:
                    if left[l]:
                        left[l] = max(0, left[l] - r)
                        if left[l] == 0:
                            finishing.setdefault(m, []).append(l)
                continue
            if in_flight:
                m, r = in_flight[0]
                t_dev = b.mark_done(m)
                if t_dev is None:
                    time.sleep(0.0002)
                    continue
                in_flight.popleft()
                if t_dev > last_mark_time[0]:
                    rate = 0.7 * rate + 0.3 * r / max((t_dev - last_mark_time[0]) * 1e3, 1e-3)
                last_mark_time = (t_dev, r)
                for l in finishing.pop(m, []):
                    job = running.pop(l)
                    left.pop(l)
                    job.done = t_origin + t_dev
                    n_samples = job.sweeps // self.measure_every if self.measure_every else 0
                    job.result = _result(b.samples_finished(l, max(n_samples, 1)), job.L, job.T, self.discard)
                    finished.append(l)
                continue
            if pending and not running:
                time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.005)))
        release_finished()
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
