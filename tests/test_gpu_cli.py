"""The Ising2D command line program of the nvidia_gpu target against the reference's own Ising2D
output (ising/src/ising_2d.cpp, recorded in tests/golden/ising2d_cli.json: hot start, 1000
warm-up sweeps, a measurement every 10 sweeps, tile 16 x 8, one lcg32 stream of 16 lanes per
tile).  Same tile and lane count through TILE_SIZE_X / TILE_SIZE_Y / LCG32_WIDTH, so the printed
energy, heat capacity and magnetisation must be the same numbers."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "computational_physics_b200", "lib", "Ising2D")
KEYS = ("Internal energy per spin", "Heat capacity per spin", "Absolute Magnetization per spin")


def _printed(stdout: str) -> dict:
    out = {}
    for line in stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            out[k.strip()] = v.strip()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("run", json.load(open(os.path.join(ROOT, "tests", "golden", "ising2d_cli.json"))),
                         ids=lambda r: f"L{r['L']}")
def test_cli_prints_reference_numbers(gpu, run):
    assert os.path.exists(CLI), "build the native library first (python -m computational_physics_b200.build)"
    L, tx, ty = run["L"], run["tile"][0], run["tile"][1]
    env = dict(os.environ, TILE_SIZE_X=str(tx), TILE_SIZE_Y=str(ty), LCG32_WIDTH="16")
    r = subprocess.run([CLI, f"--extent={L}x{L}", f"--num_sweeps={run['num_sweeps']}"], capture_output=True,
                       text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    got = _printed(r.stdout)
    for k in KEYS:
        assert got[k] == run["printed"][k], (k, got[k], run["printed"][k])
    assert got["Update time per spin"].endswith(" ns")
