"""The 3D sweep on the GPU (swb3_*) against the 3D restatement (oracle/sw_oracle.c, pinned in
tests/test_oracle3.py): bonds, resolved labels, flipped spins and lcg32 streams bit for bit,
ragged tiles and blocks included; a one-layer lattice against the 2D engine; the measurement."""
import numpy as np
import pytest

from oracle import num_tiles

pytestmark = pytest.mark.gpu


def _ntiles3(shape, tile):
    L2, L1, L0 = shape
    return num_tiles(L0, L1, tile[0], tile[1]) * -(-L2 // tile[2])


CASES = [
    # (L0, L1, L2, tile, W, T, sweeps)
    (64, 32, 16, (16, 4, 4), 16, 4.5115, 3),     # near the 3D critical temperature
    (96, 40, 12, (16, 4, 4), 16, 4.0, 2),        # ragged blocks in every direction
    (34, 18, 10, (8, 4, 2), 8, 5.0, 3),          # ragged tiles
    (32, 16, 8, (32, 2, 8), 32, 3.5, 2),
    (16, 8, 2, (16, 8, 1), 16, 4.5, 4),
    (2, 2, 2, (8, 1, 1), 16, 4.5, 3),
    (128, 128, 128, (16, 4, 4), 16, 4.5115, 2),
]


@pytest.mark.parametrize("L0,L1,L2,tile,W,T,sweeps", CASES)
def test_3d_sweeps_bit_exact_vs_oracle(gpu, oracle, L0, L1, L2, tile, W, T, sweeps):
    shape = (L2, L1, L0)
    rng = np.random.default_rng(L0 * L1 + L2)
    spins = rng.integers(0, 2, shape, dtype=np.uint8)
    r = oracle.rng_init(W, _ntiles3(shape, tile), 1)
    with gpu.SwendsenWang3D(L0, L1, L2, tile, W, 1) as sw:
        sw.set_spins(spins)
        for _ in range(sweeps - 1):
            oracle.sweep3(spins, tile, r, T=T)
        sw.update(T, sweeps - 1)
        bonds, lab = oracle.sweep3(spins, tile, r, T=T, dumps=True)
        gb, gl = sw.update_dumped(T)
        assert np.array_equal(gb, bonds)
        assert np.array_equal(gl, lab)
        assert np.array_equal(sw.get_spins(), spins)
        st, a, c, it = sw.get_rng()
        assert np.array_equal(st, r.state) and np.array_equal(it, r.iteration)
        assert np.array_equal(a, r.a) and np.array_equal(c, r.c)
        assert sw.energy_magnetization_sums() == oracle.energy_magnetization3(spins)


def test_one_layer_equals_the_2d_engine(gpu, oracle):
    """A one-layer 3D lattice's first sweep is the 2D engine's sweep of the same spins."""
    L0, L1, T = 128, 64, 2.2691853
    spins = oracle.hot_start(L0, L1, 1)
    with gpu.SwendsenWang3D(L0, L1, 1, (16, 8, 1), 16, 1) as s3, gpu.SwendsenWang2D(L0, L1, (16, 8), 16, 1) as s2:
        s3.set_spins(spins.reshape(1, L1, L0))
        s2.set_spins(spins)
        _, l3 = s3.update_dumped(T)
        _, _, l2 = s2.update_dumped(T)
        assert np.array_equal(l3[0], l2)
        assert np.array_equal(s3.get_spins()[0], s2.get_spins())


def test_3d_hot_start_and_measurement(gpu, oracle):
    L0, L1, L2, tile = 32, 32, 32, (16, 4, 4)
    with gpu.SwendsenWang3D(L0, L1, L2, tile, 16, 7) as sw:
        sw.hot_start(1)
        spins = sw.get_spins()
        assert np.array_equal(spins.reshape(L1 * L2, L0), oracle.hot_start(L0, L1 * L2, 1))
        r = oracle.rng_init(16, _ntiles3(spins.shape, tile), 7)
        sw.update(4.5, 30, measure_every=10)
        samples, acc = sw.samples()
    want = []
    for k in range(30):
        oracle.sweep3(spins, tile, r, T=4.5)
        if (k + 1) % 10 == 0:
            want.append(oracle.energy_magnetization3(spins))
    assert [tuple(x) for x in samples] == want
    assert acc[3] == 3 and acc[0] == pytest.approx(sum(-e / spins.size for e, _ in want), abs=1e-12)


def test_3d_errors(gpu):
    with pytest.raises(gpu.NativeError, match="even extents"):
        gpu.SwendsenWang3D(31, 32, 32)
    with pytest.raises(gpu.NativeError, match="tile"):
        gpu.SwendsenWang3D(32, 32, 32, (12, 4, 4))
