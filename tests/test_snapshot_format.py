"""The on-disk snapshot format (computational_physics_b200/snapshot.py) on the CPU: a chain
saved after some sweeps and resumed from the file continues exactly as the uninterrupted chain
(the oracle supplies the chain; the GPU resume is covered by the batched GPU tests)."""
import numpy as np
import pytest

from computational_physics_b200 import snapshot
from oracle import RngTiles, num_tiles

T = 2.2691853


def _chain(oracle, L0, L1, tile, W, sweeps):
    spins = oracle.hot_start(L0, L1, 1)
    rng = oracle.rng_init(W, num_tiles(L0, L1, *tile), 1)
    for _ in range(sweeps):
        oracle.sweep(spins, tile[0], tile[1], rng, T=T)
    return spins, rng


@pytest.mark.parametrize("L0,L1,tile,W", [(96, 64, (16, 8), 16), (130, 34, (8, 8), 8), (64, 64, (32, 4), 32)])
def test_resumed_chain_equals_uninterrupted(oracle, tmp_path, L0, L1, tile, W):
    spins, rng = _chain(oracle, L0, L1, tile, W, 3)
    path = str(tmp_path / "snap.npz")
    snapshot.save(path, {"L0": L0, "L1": L1, "tile": tile, "lcg_width": W, "sweeps_done": 3, "spins": spins,
                         "rng_state": rng.state, "rng_a": rng.a, "rng_c": rng.c, "rng_iteration": rng.iteration})
    snap = snapshot.load(path)
    assert (snap["L0"], snap["L1"], snap["tile"], snap["lcg_width"], snap["sweeps_done"]) == (L0, L1, tile, W, 3)
    s2 = snap["spins"].copy()
    r2 = RngTiles(W, snap["rng_state"].copy(), snap["rng_a"].copy(), snap["rng_c"].copy(),
                  snap["rng_iteration"].copy())
    assert np.array_equal(s2, spins) and r2.equal(rng)
    for _ in range(4):
        oracle.sweep(s2, tile[0], tile[1], r2, T=T)
    ref_spins, ref_rng = _chain(oracle, L0, L1, tile, W, 7)
    assert np.array_equal(s2, ref_spins)
    assert r2.equal(ref_rng)


def test_load_rejects_spins_of_another_extent(tmp_path):
    path = str(tmp_path / "bad.npz")
    snapshot.save(path, {"L0": 32, "L1": 16, "tile": (16, 8), "lcg_width": 16,
                         "spins": np.zeros((32, 32), np.uint8)})
    with pytest.raises(ValueError, match="extent"):
        snapshot.load(path)


def test_path_without_suffix_round_trips(tmp_path):
    """save('job1') and load('job1') name the same file (numpy appends .npz on save)."""
    path = str(tmp_path / "job1")
    snapshot.save(path, {"L0": 32, "L1": 16, "tile": (16, 8), "lcg_width": 16,
                         "spins": np.zeros((16, 32), np.uint8)})
    assert snapshot.load(path)["L0"] == 32


def test_load_rejects_streams_of_another_width(tmp_path):
    path = str(tmp_path / "w.npz")
    z = np.zeros((8, 8), np.uint32)  # 32 x 16 with 16 x 8 tiles has 4 tiles; W = 16 wanted
    snapshot.save(path, {"L0": 32, "L1": 16, "tile": (16, 8), "lcg_width": 16, "spins": np.zeros((16, 32), np.uint8),
                         "rng_state": z, "rng_a": z, "rng_c": z, "rng_iteration": np.zeros(4, np.uint32)})
    with pytest.raises(ValueError, match="rng_state"):
        snapshot.load(path)
