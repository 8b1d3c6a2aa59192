"""Continuous batching: jobs that share the GPU give the same results as alone, the HBM budget
gates admission, and every admitted job finishes at exactly its sweep count."""
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
