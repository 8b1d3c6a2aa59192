"""The 3D restatement (oracle/sw_oracle.c orc3_*) on the CPU: a one-layer lattice reproduces the
2D restatement's sweep (which the reference's own dumps pin), and the two bond-probability
limits have the clusters the algorithm must give: no bonds at p = 0, every aligned pair bonded
at p = 1."""
import numpy as np
import pytest

from oracle import num_tiles


def _ntiles3(shape, tile):
    L2, L1, L0 = shape
    return num_tiles(L0, L1, tile[0], tile[1]) * -(-L2 // tile[2])


@pytest.mark.parametrize("L0,L1,tile,W,T", [(64, 32, (16, 8), 16, 2.27), (100, 38, (16, 8), 16, 3.0),
                                            (32, 32, (32, 4), 16, 2.5), (48, 24, (8, 4), 8, 2.0)])
def test_one_layer_is_the_2d_sweep(oracle, L0, L1, tile, W, T):
    s2 = oracle.hot_start(L0, L1, 1)
    s3 = s2.copy().reshape(1, L1, L0)
    r2 = oracle.rng_init(W, num_tiles(L0, L1, *tile), 1)
    r3 = r2.copy()
    b2, _, l2 = oracle.sweep(s2, tile[0], tile[1], r2, T=T, dumps=True)
    b3, l3 = oracle.sweep3(s3, (tile[0], tile[1], 1), r3, T=T, dumps=True)
    assert np.array_equal(b3[0] & 3, b2) and np.array_equal(l3[0], l2) and np.array_equal(s3[0], s2)
    e, m = oracle.energy_magnetization(s2)
    e3, m3 = oracle.energy_magnetization3(s3)
    assert (e3, m3) == (e + L0 * L1, m)  # the z bond of a one-layer lattice joins a site to itself


def _components(spins):
    """Minimum site index of every same-spin periodic component (flood fill)."""
    L2, L1, L0 = spins.shape
    flat = spins.ravel()
    lab = np.full(flat.size, -1, np.int64)
    for s in range(flat.size):
        if lab[s] >= 0:
            continue
        stack = [s]
        lab[s] = s
        while stack:
            v = stack.pop()
            z, r = divmod(v, L0 * L1)
            y, x = divmod(r, L0)
            for dz, dy, dx in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                u = ((z + dz) % L2 * L1 + (y + dy) % L1) * L0 + (x + dx) % L0
                if lab[u] < 0 and flat[u] == flat[v]:
                    lab[u] = s
                    stack.append(u)
    return lab.reshape(spins.shape)


@pytest.mark.parametrize("shape,tile", [((4, 8, 16), (16, 4, 4)), ((6, 6, 10), (8, 4, 2))])
def test_bond_probability_limits(oracle, shape, tile):
    rng = np.random.default_rng(3)
    spins = rng.integers(0, 2, shape, dtype=np.uint8)
    # p = 0: no bonds, every site its own cluster, flipped iff its index is odd
    s = spins.copy()
    r = oracle.rng_init(16, _ntiles3(shape, tile), 1)
    b, lab = oracle.sweep3(s, tile, r, p_add=0.0, dumps=True)
    idx = np.arange(s.size, dtype=np.uint32).reshape(shape)
    assert not b.any() and np.array_equal(lab, idx) and np.array_equal(s, spins ^ (idx & 1).astype(np.uint8))
    # p = 1: every aligned neighbour pair bonded, clusters = same-spin components
    s = spins.copy()
    r = oracle.rng_init(16, _ntiles3(shape, tile), 1)
    b, lab = oracle.sweep3(s, tile, r, p_add=1.0, dumps=True)
    assert np.array_equal(lab, _components(spins))
    assert np.array_equal(s, spins ^ (lab & 1).astype(np.uint8))
