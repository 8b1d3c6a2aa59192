"""Host-side analysis: blocking errors, exact energies (product route vs the oracle's, and
vs the reference's own exact-energy program), and the serving job generator."""
import json
import os

import numpy as np
import pytest

from computational_physics_b200.analysis import (KC, binning_error, exact_energy, exact_energy_heat,
                                                 exact_energy_heat_precise, gate_energy)
from computational_physics_b200.serving import Job, latency_summary, poisson_jobs
from oracle.exact import exact_energy_heat as oracle_exact

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ar1(phi, n, seed=0):
    r = np.random.default_rng(seed)
    x = np.zeros(n)
    e = r.normal(size=n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return x


@pytest.mark.parametrize("phi", [0.0, 0.5, 0.9])
def test_binning_recovers_autocorrelation(phi):
    x = ar1(phi, 200_000, seed=int(phi * 10))
    b = binning_error(x)
    tau = 0.5 * (1 + phi) / (1 - phi)
    assert b.tau_int == pytest.approx(tau, rel=0.25)
    true_err = np.sqrt(2 * tau / len(x)) / np.sqrt(1 - phi * phi)
    assert b.error == pytest.approx(true_err, rel=0.25)


@pytest.mark.parametrize("L", [16, 64, 128, 192, 256, 512])
@pytest.mark.parametrize("T", [1.5, 2.0, 2.2691853, 2.6, 3.5])
def test_fast_exact_matches_oracle(L, T):
    e, c = exact_energy_heat(1.0 / T, L, L)
    oe, oc = oracle_exact(1.0 / T, L, L)
    assert e == pytest.approx(oe, abs=1e-12)
    assert c == pytest.approx(oc, rel=1e-8)


def test_exact_routes_agree_at_kc():
    for L in (32, 96):
        a = exact_energy_heat(KC, L, L)
        b = exact_energy_heat_precise(KC, L, L, 40)
        assert a[0] == pytest.approx(b[0], abs=1e-12) and a[1] == pytest.approx(b[1], rel=1e-8)


def test_exact_matches_reference_program():
    for r in json.load(open(os.path.join(GOLDEN, "exact_ff.json"))):
        e, c = exact_energy_heat(r["K"], r["L"], r["L"])
        assert e == pytest.approx(r["E"], abs=1e-12)
        assert c == pytest.approx(r["C"], rel=1e-5)
    assert exact_energy(1 / KC, 128) == pytest.approx(-1.419076272084983, abs=1e-12)


def test_rectangular_lattice_symmetry():
    assert exact_energy_heat(0.4, 64, 32)[0] == pytest.approx(exact_energy_heat(0.4, 32, 64)[0], abs=1e-12)


def test_gate_energy_on_synthetic_samples():
    L, T = 64, 2.5
    ex = exact_energy(T, L)
    r = np.random.default_rng(3)
    e_per_site = ex + 0.01 * r.normal(size=4000)
    samples = np.stack([np.round(-e_per_site * L * L).astype(np.int64), np.zeros(4000, np.int64)], axis=1)
    g = gate_energy(samples, L, L, T)
    assert g["pass"] and abs(g["z"]) < 3 and g["samples"] == 4000
    g2 = gate_energy(samples + np.array([[-int(0.05 * L * L), 0]]), L, L, T)
    assert not g2["pass"]


def test_poisson_jobs_shapes():
    jobs = poisson_jobs(100.0, 2000, seed=1)
    L = np.array([j.L for j in jobs])
    S = np.array([j.sweeps for j in jobs])
    T = np.array([j.T for j in jobs])
    t = np.array([j.arrival for j in jobs])
    assert np.all(L % 16 == 0) and L.min() >= 32 and L.max() <= 2048
    assert S.min() >= 1000 and S.max() <= 100000
    assert T.min() >= 1.5 and T.max() <= 3.5
    assert np.all(np.diff(t) > 0)
    assert 1 / np.mean(np.diff(t)) == pytest.approx(100.0, rel=0.1)
    assert len({j.seed for j in jobs}) == len(jobs)


def test_latency_summary():
    jobs = [Job(i, 32, 2.0, 1000, i + 1, arrival=float(i)) for i in range(100)]
    for j in jobs:
        j.done = j.arrival + 0.5 + 0.01 * j.jid
    s = latency_summary(jobs)
    assert s["jobs"] == 100 and s["p50_s"] == pytest.approx(0.995, abs=0.01)
    assert s["p99_s"] == pytest.approx(1.48, abs=0.02)
