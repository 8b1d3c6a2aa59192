"""The reference's own Ising2D program, built with the nvidia_gpu target plugged into its device
seams (computational_physics_b200/dropin/build_dropin.py), against the output of the
unmodified reference Ising2D (ising/src/ising_2d.cpp, recorded in tests/golden/ising2d_cli.json:
hot start, 1000 warm-up sweeps, a measurement every 10 sweeps, tile 16 x 8, one lcg32 stream of
16 lanes per tile, i.e. NUM_THREADS = number of tiles).  With the same tile, --target=nvidia_gpu
must print the same energy, heat capacity and magnetisation, digit for digit, as the recording
and as --target=cpu of the same binary.  The recordings include a sweep count that is not a
multiple of 10 and the CPU configuration's full protocol (128 x 128, 100000 sweeps)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "computational_physics_b200", "lib", "dropin", "Ising2D")
KEYS = ("Internal energy per spin", "Heat capacity per spin", "Absolute Magnetization per spin")
RUNS = json.load(open(os.path.join(ROOT, "tests", "golden", "ising2d_cli.json")))


def _printed(stdout: str) -> dict:
    out = {}
    for line in stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            out[k.strip()] = v.strip()
    return out


def _run(run, target, timeout=600):
    if not os.path.exists(CLI):
        pytest.fail("the drop-in Ising2D is missing: python -m computational_physics_b200.dropin.build_dropin")
    L, tx, ty = run["L"], run["tile"][0], run["tile"][1]
    env = dict(os.environ, TILE_SIZE_X=str(tx), TILE_SIZE_Y=str(ty), NUM_THREADS=str(run["NUM_THREADS"]))
    r = subprocess.run([CLI, f"--target={target}", f"--extent={L}x{L}", f"--num_sweeps={run['num_sweeps']}"],
                       capture_output=True, text=True, timeout=timeout, env=env)
    assert r.returncode == 0, r.stderr
    return _printed(r.stdout)


@pytest.mark.parametrize("run", [r for r in RUNS if r["L"] ** 2 * r["num_sweeps"] <= 64 * 64 * 1000],
                         ids=lambda r: f"L{r['L']}x{r['num_sweeps']}")
def test_dropin_cpu_target_is_the_reference(run):
    """The drop-in binary's CPU target is the reference's unchanged CPU path (no GPU needed)."""
    got = _run(run, "cpu")
    assert got["Target name"] == "CPU"
    for k in KEYS:
        assert got[k] == run["printed"][k], (k, got[k], run["printed"][k])


@pytest.mark.gpu
@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"L{r['L']}x{r['num_sweeps']}")
def test_dropin_gpu_target_prints_reference_numbers(gpu, run):
    got = _run(run, "nvidia_gpu")
    assert got["Target name"] == "NVIDIA GPU"
    for k in KEYS:
        assert got[k] == run["printed"][k], (k, got[k], run["printed"][k])
    assert got["Update time per spin"].endswith(" ns")
    if run["L"] ** 2 * run["num_sweeps"] <= 64 * 64 * 1000:
        cpu = _run(run, "cpu")
        for k in KEYS:
            assert got[k] == cpu[k], (k, got[k], cpu[k])


@pytest.mark.gpu
def test_dropin_rejects_odd_extent(gpu):
    r = subprocess.run([CLI, "--target=nvidia_gpu", "--extent=31x32", "--num_sweeps=10"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0
    assert "evenly sized" in r.stderr
