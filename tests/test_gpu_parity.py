"""Bit-exact parity of the CUDA sweep with the reference, through the C ABI.

Small cases compare against the committed dumps of the unmodified reference
(tests/golden/); larger ones against the C restatement (oracle/), which those dumps pin;
the largest ones through size-independent invariants."""
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


@pytest.mark.parametrize("resolve_min", ["1", "1000000000"])
@pytest.mark.parametrize("L0,L1,tile,W,T,sweeps", [CASES[0], CASES[3], CASES[4], CASES[7]])
def test_resolve_kernel_and_chasing_flip_agree_with_oracle(gpu, oracle, monkeypatch, resolve_min, L0, L1, tile, W, T,
                                                          sweeps):
    """Merged roots resolved by their own kernel (threshold 1 block) or chased by the flip
    (threshold above any lattice): both bit-exact with the oracle, stage dumps included."""
    monkeypatch.setenv("SWB_RESOLVE_MIN_BLOCKS", resolve_min)
    test_sweeps_bit_exact_vs_oracle(gpu, oracle, L0, L1, tile, W, T, sweeps)


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


def test_invariants_at_16384(gpu):
    """Size-independent properties at the bandwidth config's largest lattice: labels are
    roots and minimal (label <= site index, label[label] == label), every bond joins equal
    spins, flipping follows the label parity, and a resweep is deterministic."""
    L = 16384
    with gpu.SwendsenWang2D(L, L, (16, 8), 16) as sw:
        sw.hot_start(1)
        sw.update(2.2691853, 2)
        before = sw.get_spins()
        bonds, la, lf = sw.update_recorded(2.2691853)
        after = sw.get_spins()
    flat = lf.ravel()
    R = 512
    for y0 in range(0, L, R):
        rows = slice(y0, y0 + R)
        idx = np.arange(y0 * L, (y0 + R) * L, dtype=np.uint32).reshape(R, L)
        f = lf[rows]
        assert np.all(f <= idx)
        assert np.array_equal(flat[f.ravel()], f.ravel())
        assert np.all(la[rows] >= f)
        down = np.concatenate([lf[y0 + 1:y0 + R], lf[(y0 + R) % L][None]])
        sdown = np.concatenate([before[y0 + 1:y0 + R], before[(y0 + R) % L][None]])
        b = bonds[rows]
        s = before[rows]
        xb = (b & 1).astype(bool)
        yb = (b & 2).astype(bool)
        assert np.all(s[xb] == np.roll(s, -1, axis=1)[xb])
        assert np.all(s[yb] == sdown[yb])
        assert np.all(f[xb] == np.roll(f, -1, axis=1)[xb])
        assert np.all(f[yb] == down[yb])
        assert np.array_equal(after[rows], s ^ (f & 1).astype(np.uint8))


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
