"""Host logic of the continuous-batching server (computational_physics_b200/serving.py) on the
CPU, with a stand-in for the batched engine: admission under the HBM budget and the slot
limit, back-pressure while the GPU is full, rejection of a job too big for an empty GPU,
completion bookkeeping and the latency summary.  The GPU serving run is tests/test_gpu_serving.py."""
import numpy as np
import pytest

from computational_physics_b200 import serving
from computational_physics_b200._native import NativeError
from computational_physics_b200.analysis import exact_energy


class FakeBatch:
    """BatchedSW's calls the server makes: `capacity` slots, a budget of L * L per lattice, the
    sweep budgets counted down per round and one (e, m) sample per measure_every sweeps, spread
    by +-4 around the exact energy."""

    def __init__(self, capacity, budget, lcg_width=16, device=0):
        self.capacity, self.budget = capacity, budget
        self.rounds = 0
        self.lat = {}
        self.max_used = 0
        self.max_running = 0

    def used(self):
        return sum(v["L"] ** 2 for v in self.lat.values())

    def add(self, L0, L1, temperature, seed_base, tile, block):
        free = [i for i in range(self.capacity) if i not in self.lat]
        if not free or self.used() + L0 * L1 > self.budget:
            raise NativeError(4, "no slot or budget left")
        lid = free[0]
        self.lat[lid] = {"L": L0, "T": temperature, "left": 0, "every": 0, "done": 0, "samples": []}
        self.max_used = max(self.max_used, self.used())
        self.max_running = max(self.max_running, len(self.lat))
        return lid

    def hot_start(self, lid, seed):
        assert lid in self.lat

    def set_schedule(self, lid, sweeps, measure_every):
        self.lat[lid].update(left=sweeps, every=measure_every)

    def sweep(self, rounds=1, measure=False):
        self.rounds += rounds
        for v in self.lat.values():
            for _ in range(min(rounds, v["left"])):
                v["left"] -= 1
                v["done"] += 1
                if measure and v["every"] and v["done"] % v["every"] == 0:
                    n = v["L"] ** 2
                    e = round(-exact_energy(v["T"], v["L"]) * n) + (4 if len(v["samples"]) % 2 else -4)
                    v["samples"].append((e, 0))

    def poll(self):
        left = np.zeros(self.capacity, np.uint32)
        done = np.zeros(self.capacity, np.uint32)
        for lid, v in self.lat.items():
            left[lid], done[lid] = v["left"], v["done"]
        return left, done

    def samples(self, lid):
        return np.array(self.lat[lid]["samples"], np.int64).reshape(-1, 2)

    def samples_finished(self, lid, max_samples):
        assert self.lat[lid]["left"] == 0, "read before the lattice finished"
        return self.samples(lid)[:max_samples]

    # device progress: the fake runs rounds at once; a mark's "device time" is 0.1 ms per round
    def mark(self):
        self.marks = getattr(self, "marks", []) + [self.rounds]
        return len(self.marks) - 1

    def mark_done(self, m):
        return 1e-4 * self.marks[m]

    def remove(self, lid):
        del self.lat[lid]

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    made = []

    def factory(capacity, budget, lcg_width=16, device=0):
        made.append(FakeBatch(capacity, budget, lcg_width, device))
        return made[-1]

    monkeypatch.setattr(serving, "BatchedSW", factory)
    monkeypatch.setattr(serving.autotune, "load", lambda *a, **k: {})
    return made


def _jobs(sides, sweeps):
    return [serving.Job(i, L, 2.2691853, s, 1 + i, arrival=0.001 * i) for i, (L, s) in enumerate(zip(sides, sweeps))]


def test_admission_respects_budget_and_every_job_completes(fake):
    jobs = _jobs([64] * 7, [200, 400, 100, 300, 500, 200, 100])
    srv = serving.Server(hbm_budget_bytes=3 * 64 * 64, capacity=8, measure_every=10)
    srv.run(jobs, realtime=False)
    eng = fake[0]
    assert eng.max_used <= 3 * 64 * 64 and eng.max_running == 3  # back-pressure, not rejection
    assert not srv.rejected and not eng.lat                        # all finished and removed
    for j in jobs:
        assert j.done is not None and j.admitted is not None and j.done >= j.admitted
        assert j.result["samples"] == j.sweeps // 10
        assert j.result["exact_E"] == pytest.approx(exact_energy(j.T, j.L))
        assert abs(j.result["E"] - j.result["exact_E"]) < 1e-3
    admitted = [j.admitted for j in sorted(jobs, key=lambda j: j.arrival)]
    assert admitted == sorted(admitted)                            # first come, first admitted


def test_bounded_bypass_of_a_head_job_that_does_not_fit(fake):
    """A big job at the head waits for memory; small jobs behind it go ahead, but only
    max_bypass of them, after which the head is served first."""
    sides = [64, 64, 128] + [32] * 6
    jobs = _jobs(sides, [400, 400, 100] + [50] * 6)
    srv = serving.Server(hbm_budget_bytes=128 * 128, capacity=8, measure_every=10, max_bypass=2)
    srv.run(jobs, realtime=False)
    assert not srv.rejected and all(j.done is not None for j in jobs)
    assert srv.bypassed == 2
    big = jobs[2]
    ahead = [j for j in jobs[3:] if j.admitted < big.admitted]
    assert len(ahead) == 2


def test_jobs_finish_in_their_own_round(fake):
    """A job's completion is the device time of the mark after its last round: with jobs of
    100, 200, 300 sweeps admitted together, 0.1 ms per round in the fake."""
    jobs = _jobs([32, 32, 32], [100, 200, 300])
    srv = serving.Server(hbm_budget_bytes=10 ** 9, capacity=4, measure_every=10, max_rounds=10 ** 6)
    srv.run(jobs, realtime=False)
    d = [j.done for j in jobs]
    assert d[1] - d[0] == pytest.approx(100 * 1e-4, abs=1e-6) and d[2] - d[1] == pytest.approx(100 * 1e-4, abs=1e-6)


def test_slot_limit_holds_back_jobs(fake):
    jobs = _jobs([32] * 5, [50] * 5)
    srv = serving.Server(hbm_budget_bytes=10 ** 9, capacity=2, measure_every=10)
    srv.run(jobs, realtime=False)
    assert fake[0].max_running == 2
    assert all(j.done is not None for j in jobs) and not srv.rejected


def test_job_too_big_for_an_empty_gpu_is_rejected(fake):
    jobs = _jobs([64, 256, 64], [100, 100, 100])
    srv = serving.Server(hbm_budget_bytes=2 * 64 * 64, capacity=4, measure_every=10)
    srv.run(jobs, realtime=False)
    assert [j.jid for j in srv.rejected] == [1]
    assert jobs[1].done is None and jobs[0].done is not None and jobs[2].done is not None


def test_latency_summary():
    jobs = [serving.Job(i, 32, 2.0, 100, 1, arrival=float(i)) for i in range(4)]
    for j, lat in zip(jobs, (1.0, 2.0, 3.0, 4.0)):
        j.done = j.arrival + lat
    s = serving.latency_summary(jobs)
    assert s["jobs"] == 4 and s["p50_s"] == pytest.approx(2.5) and s["mean_s"] == pytest.approx(2.5)
    assert s["makespan_s"] == pytest.approx(7.0)
    assert s["site_updates_per_s"] == pytest.approx(4 * 32 * 32 * 100 / 7.0)
    assert serving.latency_summary([serving.Job(0, 32, 2.0, 1, 1)]) == {"jobs": 0}


def test_autotune_choice_uses_the_nearest_tuned_side():
    from computational_physics_b200 import autotune
    table = autotune.load("NVIDIA B200")
    assert autotune.choice(64, table) == ((16, 4), (4, 8))       # the committed B200 table's entry for 64
    assert autotune.choice(70, table) == autotune.choice(64, table)
    assert autotune.choice(4096, table) == autotune.choice(512, table)
    assert autotune.choice(100, {}) == ((16, 8), (0, 0))          # no table: the default tile
    assert autotune.cache_path("NVIDIA B200", 16).endswith("tuned/nvidia_b200_w16.json")
