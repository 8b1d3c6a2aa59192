"""Bit-exact parity of the CUDA sweep with the reference, through the C ABI.

Small cases compare against the committed dumps of the unmodified reference
(tests/golden/); larger ones against the C restatement (oracle/), which those dumps pin;
the largest ones (4096^2 - 16384^2) against digests of the restatement's output
(tests/golden/c3_sha.json)."""
import hashlib

import numpy as np
import pytest

from oracle import num_tiles

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def _golden_spins(oracle, g, key, L0, L1):
    if key + "_spins_in" in g:
        return g[key + "_spins_in"].copy()
    seed, kind = (int(x) for x in g[key + "_spins_in_seed"])
    return oracle.hot_start(L0, L1, 1) if kind == 0 else \
        np.random.default_rng(seed).integers(0, 2, (L1, L0), dtype=np.uint8)


@pytest.mark.parametrize("width", [16, 8])
def test_stages_bit_exact_vs_reference_dumps(gpu, oracle, golden16, golden8, width):
    g = golden16 if width == 16 else golden8
    for k, case in enumerate(g["sw_cases"]):
        L0, L1, tx, ty, T, ns, sb = case
        L0, L1, tx, ty, ns, sb = int(L0), int(L1), int(tx), int(ty), int(ns), int(sb)
        key = f"sw{k}"
        spins = _golden_spins(oracle, g, key, L0, L1)
        with gpu.SwendsenWang2D(L0, L1, (tx, ty), width, sb) as sw:
            sw.set_spins(spins)
            if ns > 1:
                sw.update(float(T), ns - 1)
            bonds, la, lf = sw.update_recorded(float(T))
            out = sw.get_spins()
            st, a, c, it = sw.get_rng()
        if key + "_bonds" in g:
            assert np.array_equal(bonds, g[key + "_bonds"]), key
            assert np.array_equal(la, g[key + "_labels_assign"]), key
            assert np.array_equal(lf, g[key + "_labels_final"]), key
            assert np.array_equal(out, g[key + "_spins_out"]), key
            assert np.array_equal(st, g[key + "_rng_state"]), key
            assert np.array_equal(a, g[key + "_rng_a"]), key
            assert np.array_equal(c, g[key + "_rng_c"]), key
            assert np.array_equal(it, g[key + "_rng_iteration"]), key
        else:
            for name, arr in (("bonds", bonds), ("labels_assign", la), ("labels_final", lf), ("spins_out", out),
                              ("rng_state", st), ("rng_iteration", it)):
                assert sha(arr) == g[key + "_" + name + "_sha"].tobytes(), (key, name)


@pytest.mark.parametrize("width", [8, 16, 32])
def test_rng_init_matches_oracle(gpu, oracle, width):
    L0, L1, tx, ty = 256, 128, 16, 8
    with gpu.SwendsenWang2D(L0, L1, (tx, ty), width, seed_base=11) as sw:
        st, a, c, it = sw.get_rng()
    r = oracle.rng_init(width, num_tiles(L0, L1, tx, ty), 11)
    assert np.array_equal(st, r.state) and np.array_equal(a, r.a) and np.array_equal(c, r.c)
    assert np.array_equal(it, r.iteration)


@pytest.mark.parametrize("L0,L1", [(64, 32), (1024, 1024), (1000, 998)])
def test_hot_start_matches_oracle(gpu, oracle, L0, L1):
    with gpu.SwendsenWang2D(L0, L1) as sw:
        sw.hot_start(1)
        got = sw.get_spins()
    assert np.array_equal(got, oracle.hot_start(L0, L1, 1))


CASES = [
    # (L0, L1, tile, W, T, sweeps)
    (1024, 1024, (8, 8), 16, 2.2691853, 3),    # the single-lattice GPU config
    (128, 128, (16, 8), 16, 2.2691853, 20),    # the CPU config
    (512, 384, (16, 8), 8, 2.0, 4),
    (640, 200, (32, 4), 16, 3.0, 3),
    (258, 130, (16, 8), 16, 2.2691853, 4),     # ragged tiles and blocks
    (2048, 64, (8, 16), 32, 2.5, 2),
    (32, 4096, (16, 32), 16, 1.8, 2),
    (2, 2, (16, 8), 16, 2.2691853, 5),
    (2048, 2048, (16, 8), 16, 2.2691853, 2),
]


@pytest.mark.parametrize("L0,L1,tile,W,T,sweeps", CASES)
def test_sweeps_bit_exact_vs_oracle(gpu, oracle, L0, L1, tile, W, T, sweeps):
    spins = oracle.hot_start(L0, L1, 1)
    rng = oracle.rng_init(W, num_tiles(L0, L1, *tile), 1)
    with gpu.SwendsenWang2D(L0, L1, tile, W, 1) as sw:
        sw.set_spins(spins)
        for s in range(sweeps - 1):
            oracle.sweep(spins, tile[0], tile[1], rng, T=T)
        sw.update(T, sweeps - 1)
        bonds, la, lf = oracle.sweep(spins, tile[0], tile[1], rng, T=T, dumps=True)
        gb, gla, glf = sw.update_recorded(T)
        assert np.array_equal(gb, bonds)
        assert np.array_equal(gla, la)
        assert np.array_equal(glf, lf)
        assert np.array_equal(sw.get_spins(), spins)
        st, a, c, it = sw.get_rng()
        assert np.array_equal(st, rng.state) and np.array_equal(it, rng.iteration)
        e, m = oracle.energy_magnetization(spins)
        assert sw.energy_magnetization_sums() == (e, m)


@pytest.mark.parametrize("L0,L1,tile,W,T,sweeps", CASES)
def test_production_sweep_bit_exact_vs_oracle(gpu, oracle, L0, L1, tile, W, T, sweeps):
    """The kernels a plain sweep runs, with their dumps on: bonds, the labels over the bonds
    inside each assign block, resolved labels, flipped spins and lcg32 streams."""
    spins = oracle.hot_start(L0, L1, 1)
    rng = oracle.rng_init(W, num_tiles(L0, L1, *tile), 1)
    with gpu.SwendsenWang2D(L0, L1, tile, W, 1) as sw:
        geo = sw.geometry()
        sw.set_spins(spins)
        for s in range(sweeps - 1):
            oracle.sweep(spins, tile[0], tile[1], rng, T=T)
        sw.update(T, sweeps - 1)
        bonds, _, lf = oracle.sweep(spins, tile[0], tile[1], rng, T=T, dumps=True)
        gb, glb, glf = sw.update_dumped(T)
        assert np.array_equal(gb, bonds)
        assert np.array_equal(glb, oracle.block_labels(bonds, geo["block_x"], geo["block_y"]))
        assert np.array_equal(glf, lf)
        assert np.array_equal(sw.get_spins(), spins)
        st, a, c, it = sw.get_rng()
        assert np.array_equal(st, rng.state) and np.array_equal(it, rng.iteration)
        assert np.array_equal(a, rng.a) and np.array_equal(c, rng.c)


@pytest.mark.parametrize("L", [4096, 8192, 16384])
def test_bandwidth_sizes_bit_exact(gpu, c3_fixtures, L):
    """4096^2 - 16384^2 (tile 16 x 8, W = 16, hot start, T_c): the third sweep of the kernels a
    plain sweep runs, digest for digest against the CPU restatement (tests/golden/c3_sha.json;
    the 4096^2 digests also agree with the unmodified reference sources)."""
    fx = c3_fixtures
    want = fx["cases"][str(L)]
    T = fx["temperature"]
    with gpu.SwendsenWang2D(L, L, tuple(fx["tile"]), fx["lcg_width"], fx["seed_base"]) as sw:
        geo = sw.geometry()
        sw.hot_start(fx["hot_start_seed"])
        sw.update(T, fx["sweeps_before"])
        assert sha(sw.get_spins()).hex() == want["spins_in"]
        bonds, lb, lf = sw.update_dumped(T)
        assert sha(bonds).hex() == want["bonds"]
        del bonds
        if [geo["block_x"], geo["block_y"]] == fx["block"]:
            assert sha(lb).hex() == want["labels_block"]
        del lb
        assert sha(lf).hex() == want["labels_final"]
        del lf
        assert sha(sw.get_spins()).hex() == want["spins_out"]
        st, _, _, it = sw.get_rng()
        assert sha(st).hex() == want["rng_state"]
        assert sha(it).hex() == want["rng_iteration"]


@pytest.mark.parametrize("resolve_min", ["1", "1000000000"])
@pytest.mark.parametrize("L0,L1,tile,W,T,sweeps", [CASES[0], CASES[3], CASES[4], CASES[7]])
def test_resolve_kernel_and_chasing_flip_agree_with_oracle(gpu, oracle, monkeypatch, resolve_min, L0, L1, tile, W, T,
                                                          sweeps):
    """Merged roots resolved by their own kernel (threshold 1 block) or chased by the flip
    (threshold above any lattice): both bit-exact with the oracle, stage dumps included."""
    monkeypatch.setenv("SWB_RESOLVE_MIN_BLOCKS", resolve_min)
    test_sweeps_bit_exact_vs_oracle(gpu, oracle, L0, L1, tile, W, T, sweeps)
    test_production_sweep_bit_exact_vs_oracle(gpu, oracle, L0, L1, tile, W, T, sweeps)


def test_set_rng_roundtrip_and_continue(gpu, oracle):
    L0 = L1 = 256
    spins = oracle.hot_start(L0, L1, 1)
    rng = oracle.rng_init(16, num_tiles(L0, L1, 16, 8), 1)
    for _ in range(7):
        oracle.sweep(spins, 16, 8, rng, T=2.2691853)
    with gpu.SwendsenWang2D(L0, L1, (16, 8), 16, seed_base=999) as sw:
        sw.set_spins(spins)
        sw.set_rng(rng.state, rng.a, rng.c, rng.iteration)
        sw.update(2.2691853, 5)
        for _ in range(5):
            oracle.sweep(spins, 16, 8, rng, T=2.2691853)
        assert np.array_equal(sw.get_spins(), spins)


def test_errors_are_reported(gpu):
    with pytest.raises(gpu.NativeError, match="evenly sized"):
        gpu.SwendsenWang2D(31, 32)
    with gpu.SwendsenWang2D(32, 32) as sw:
        with pytest.raises(gpu.NativeError, match="0 or 1"):
            sw.set_spins(np.full((32, 32), 2, np.uint8))
        with pytest.raises(gpu.NativeError, match="temperature"):
            sw.update(-1.0)
        sw.update(2.0, 2)   # the handle stays usable


def test_measurement_accumulators(gpu, oracle):
    L = 64
    spins = oracle.hot_start(L, L, 1)
    rng = oracle.rng_init(16, num_tiles(L, L, 16, 8), 1)
    with gpu.SwendsenWang2D(L, L, (16, 8), 16) as sw:
        sw.set_spins(spins)
        sw.update(2.2691853, 40, measure_every=10)
        acc = sw.accumulators()
        samples = sw.samples()
    E = []
    M = []
    for k in range(40):
        oracle.sweep(spins, 16, 8, rng, T=2.2691853)
        if (k + 1) % 10 == 0:
            e, m = oracle.energy_magnetization(spins)
            E.append(-e / (L * L))
            M.append(abs(m) / (L * L))
            assert tuple(samples[len(E) - 1]) == (e, m)
    assert acc[3] == 4
    assert acc[0] == pytest.approx(sum(E), abs=1e-12)
    assert acc[1] == pytest.approx(sum(x * x for x in E), abs=1e-12)
    assert acc[2] == pytest.approx(sum(M), abs=1e-12)


@pytest.mark.parametrize("L0,L1,tile", [(256, 128, (16, 8)), (8, 64, (8, 8)), (200, 96, (8, 8))])
def test_measurement_taken_by_the_next_sweep(gpu, oracle, L0, L1, tile):
    """Samples every 10 sweeps: the sample of the spins after sweep k is taken by sweep k + 1's
    assign phase (no k_measure launch while sweeps follow), the last one when the observables are
    read; all exact.  The 8-wide lattice's blocks are narrower than a 32-site word, so there
    every sample is taken by k_measure."""
    spins = oracle.hot_start(L0, L1, 1)
    rng = oracle.rng_init(16, num_tiles(L0, L1, *tile), 1)
    with gpu.SwendsenWang2D(L0, L1, tile, 16) as sw:
        sw.set_spins(spins)
        fused = sw.geometry()["block_x"] % 32 == 0
        n0 = gpu.kernel_launches()
        sw.update(2.2691853, 40, measure_every=10)
        launched = gpu.kernel_launches() - n0
        samples = sw.samples()
        acc = sw.accumulators()
        per_sweep = sw.launches_per_sweep()
    assert launched == 40 * per_sweep + (0 if fused else 3)
    want = []
    for k in range(40):
        oracle.sweep(spins, tile[0], tile[1], rng, T=2.2691853)
        if (k + 1) % 10 == 0:
            want.append(oracle.energy_magnetization(spins))
    assert [tuple(x) for x in samples] == want
    E = [-e / (L0 * L1) for e, _ in want]
    assert acc[3] == 4 and acc[0] == pytest.approx(sum(E), abs=1e-12)


def test_update_host_matches_device_path(gpu, oracle):
    L = 256
    spins = oracle.hot_start(L, L, 1)
    out = np.empty_like(spins)
    em = np.zeros(2)
    with gpu.SwendsenWang2D(L, L, (8, 8), 16) as a, gpu.SwendsenWang2D(L, L, (8, 8), 16) as b:
        a.update_host(2.2691853, spins, out, em)
        b.set_spins(spins)
        b.update(2.2691853)
        assert np.array_equal(out, b.get_spins())
        assert tuple(em) == b.energy_magnetization()
