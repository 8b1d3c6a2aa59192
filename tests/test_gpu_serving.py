"""Continuous batching: jobs that share the GPU give the same results as alone and as the CPU
restatement of the reference, the HBM budget gates admission, and every admitted job finishes at
exactly its sweep count."""
import numpy as np
import pytest

from computational_physics_b200.batch import lattice_bytes
from computational_physics_b200.serving import Job, SequentialServer, Server, latency_summary, poisson_jobs

pytestmark = pytest.mark.gpu


def small_jobs(n=12, seed=5):
    js = poisson_jobs(1000.0, n, seed=seed, L_range=(32, 256), sweeps_range=(100, 600))
    return js


def test_results_same_alone_and_in_mix(gpu):
    jobs = small_jobs()
    mixed = Server(hbm_budget_bytes=0, capacity=64)
    mixed.run(jobs, realtime=False)
    mixed.close()
    for j in jobs:
        assert j.done is not None and j.result["samples"] == j.sweeps // 10
        solo = Job(j.jid, j.L, j.T, j.sweeps, j.seed)
        s = Server(hbm_budget_bytes=0, capacity=1)
        s.run([solo], realtime=False)
        s.close()
        assert np.array_equal(solo.result.pop("series"), j.result.pop("series")), j
        assert solo.result == j.result, j


def test_sequential_baseline_agrees(gpu):
    jobs = small_jobs(6, seed=9)
    seq = [Job(j.jid, j.L, j.T, j.sweeps, j.seed, j.arrival) for j in jobs]
    srv = Server(hbm_budget_bytes=0, capacity=16)
    srv.run(jobs, realtime=False)
    srv.close()
    SequentialServer().run(seq, realtime=False)
    for a, b in zip(sorted(jobs, key=lambda j: j.jid), sorted(seq, key=lambda j: j.jid)):
        assert a.result["E"] == b.result["E"] and a.result["absM"] == b.result["absM"]


def test_budget_admission_and_rejection(gpu):
    big = lattice_bytes(256, 256)
    jobs = [Job(i, 256, 2.3, 200, 10 + i) for i in range(5)] + [Job(99, 1024, 2.3, 100, 3)]
    srv = Server(hbm_budget_bytes=int(big * 2.5), capacity=8)
    srv.run(jobs, realtime=False)
    srv.close()
    done = [j for j in jobs if j.done is not None]
    assert len(done) == 5                       # two at a time fit; all five finish
    assert [j.jid for j in srv.rejected] == [99]  # larger than the whole budget


def test_realtime_poisson_latency(gpu):
    jobs = poisson_jobs(200.0, 24, seed=2, L_range=(32, 192), sweeps_range=(200, 1000))
    srv = Server(hbm_budget_bytes=0, capacity=64)
    srv.run(jobs, realtime=True)
    srv.close()
    s = latency_summary(jobs)
    assert s["jobs"] == 24 and s["p99_s"] >= s["p50_s"] > 0
    assert all(np.isfinite(j.result["E"]) for j in jobs)


def test_served_series_equal_the_oracle(gpu, oracle):
    """Jobs served together: each job's recorded (e, m) integer series is the restatement's for
    that job alone (hot start and lcg32 streams from the job's seed, the served tile)."""
    from computational_physics_b200 import autotune
    from oracle import num_tiles
    jobs = [Job(0, 32, 2.1, 120, 7), Job(1, 48, 2.6, 200, 8), Job(2, 64, 2.27, 90, 9), Job(3, 96, 3.0, 150, 10)]
    srv = Server(hbm_budget_bytes=0, capacity=8, measure_every=10)
    srv.run(jobs, realtime=False)
    srv.close()
    table = autotune.load()
    for j in jobs:
        tile, _ = autotune.choice(j.L, table)
        spins = oracle.hot_start(j.L, j.L, j.seed)
        rng = oracle.rng_init(16, num_tiles(j.L, j.L, *tile), j.seed)
        want = []
        for k in range(j.sweeps):
            oracle.sweep(spins, tile[0], tile[1], rng, T=j.T)
            if (k + 1) % 10 == 0:
                want.append(oracle.energy_magnetization(spins))
        assert [tuple(x) for x in j.result["series"]] == want, j.jid
