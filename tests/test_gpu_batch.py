"""The batched engine: every lattice of a mix is bit-identical to the reference path for its
extent, tile, lcg width and seeds, whatever else shares the GPU."""
import numpy as np
import pytest

from oracle import num_tiles

pytestmark = pytest.mark.gpu

MIX = [
    # (L0, L1, tile, T, seed_base, block)
    (64, 64, (16, 8), 2.2691853, 1, (0, 0)),
    (96, 96, (8, 8), 2.1, 7, (0, 0)),
    (128, 128, (16, 8), 2.5, 3, (4, 2)),
    (192, 64, (32, 4), 2.0, 11, (0, 0)),
    (48, 256, (8, 16), 2.6, 5, (2, 2)),
    (100, 38, (16, 8), 3.0, 2, (0, 0)),     # ragged tiles
    (2, 2, (16, 8), 2.2691853, 9, (0, 0)),
    (512, 512, (16, 8), 2.3, 13, (0, 0)),
]

# Only the tiles the lean batched assign instance compiles (16 x 8 and 16 x 4) or neither
# instance does (16 x 2, the runtime path): the engine launches the lean instance.
LEAN_MIX = [
    (64, 64, (16, 4), 2.2691853, 21, (0, 0)),
    (96, 96, (16, 8), 2.1, 22, (0, 0)),
    (128, 128, (16, 8), 2.5, 23, (4, 2)),
    (100, 38, (16, 8), 3.0, 24, (0, 0)),     # ragged tiles
    (64, 32, (16, 2), 2.4, 25, (0, 0)),
    (384, 384, (16, 8), 2.3, 26, (0, 0)),
]


def _oracle_run(oracle, spins, tile, T, seed, sweeps, W=16):
    L1, L0 = spins.shape
    rng = oracle.rng_init(W, num_tiles(L0, L1, *tile), seed)
    s = spins.copy()
    for _ in range(sweeps):
        oracle.sweep(s, tile[0], tile[1], rng, T=T)
    return s, rng


@pytest.mark.parametrize("mix", [MIX, LEAN_MIX], ids=["all_shapes", "lean"])
def test_mix_bit_exact(gpu, oracle, mix):
    rounds = 6
    with gpu.BatchedSW(capacity=64) as b:
        ids, starts = [], []
        for k, (L0, L1, tile, T, seed, block) in enumerate(mix):
            i = b.add(L0, L1, T, seed, tile, block)
            start = oracle.hot_start(L0, L1, 1) if k % 2 == 0 else \
                np.random.default_rng(k).integers(0, 2, (L1, L0), dtype=np.uint8)
            b.set_spins(i, start)
            ids.append(i)
            starts.append(start)
        b.sweep(rounds)
        b.synchronize()
        for i, start, (L0, L1, tile, T, seed, block) in zip(ids, starts, mix):
            want, rng = _oracle_run(oracle, start, tile, T, seed, rounds)
            assert np.array_equal(b.get_spins(i), want), (L0, L1, tile)
            st, a, c, it = b.get_rng(i)
            assert np.array_equal(st, rng.state) and np.array_equal(it, rng.iteration)


def test_schedules_and_alone_vs_mix(gpu, oracle):
    """A lattice with a 3-sweep budget stops after 3 sweeps while the rest continue; the
    same lattice alone in its own batch ends in the same state."""
    with gpu.BatchedSW(capacity=16) as mix, gpu.BatchedSW(capacity=2) as alone:
        a = mix.add(128, 128, 2.2691853, 1, (16, 8))
        others = [mix.add(L, L, 2.4, 100 + L, (8, 8)) for L in (64, 256, 96)]
        solo = alone.add(128, 128, 2.2691853, 1, (16, 8))
        for lid in [a, *others]:
            mix.hot_start(lid, 1)
        alone.hot_start(solo, 1)
        mix.set_schedule(a, 3, 1)
        alone.set_schedule(solo, 3, 1)
        mix.sweep(5, measure=True)
        alone.sweep(3, measure=True)
        mix.synchronize()
        assert mix.status(a) == (0, 3)
        assert mix.status(others[0])[1] == 5
        got = mix.get_spins(a)
        assert np.array_equal(got, alone.get_spins(solo))
        want, _ = _oracle_run(oracle, oracle.hot_start(128, 128, 1), (16, 8), 2.2691853, 1, 3)
        assert np.array_equal(got, want)
        s_mix = mix.samples(a)
        assert np.array_equal(s_mix, alone.samples(solo))
        assert len(s_mix) == 3


def test_measurement_matches_oracle(gpu, oracle):
    L, T = 96, 2.2691853
    with gpu.BatchedSW(capacity=4) as b:
        i = b.add(L, L, T, 1, (16, 8))
        b.hot_start(i, 1)
        b.set_schedule(i, 40, 10)
        b.sweep(40, measure=True)
        acc = b.accumulators(i)
        samples = b.samples(i)
    s = oracle.hot_start(L, L, 1)
    rng = oracle.rng_init(16, num_tiles(L, L, 16, 8), 1)
    E = []
    for k in range(40):
        oracle.sweep(s, 16, 8, rng, T=T)
        if (k + 1) % 10 == 0:
            e, m = oracle.energy_magnetization(s)
            assert tuple(samples[len(E)]) == (e, m)
            E.append(-e / (L * L))
    assert acc[3] == 4 and acc[0] == pytest.approx(sum(E), abs=1e-12)


def test_add_remove_between_rounds(gpu, oracle):
    with gpu.BatchedSW(capacity=8) as b:
        x = b.add(64, 64, 2.3, 1, (16, 8))
        b.hot_start(x, 1)
        b.sweep(2)
        y = b.add(128, 64, 2.0, 4, (8, 8))
        b.hot_start(y, 1)
        b.sweep(3)
        b.remove(x)
        b.sweep(2)
        got_y = b.get_spins(y)
    want_y, _ = _oracle_run(oracle, oracle.hot_start(128, 64, 1), (8, 8), 2.0, 4, 5)
    assert np.array_equal(got_y, want_y)


def test_hbm_budget_admission(gpu):
    need = gpu.lattice_bytes(512, 512, (16, 8))
    with gpu.BatchedSW(capacity=8, hbm_budget_bytes=int(need * 2.5)) as b:
        b.add(512, 512)
        b.add(512, 512)
        with pytest.raises(gpu.NativeError, match="bytes"):
            b.add(512, 512)
        used, budget = b.memory()
        assert used == 2 * need and budget == int(need * 2.5)
    with gpu.BatchedSW(capacity=1) as b:
        b.add(64, 64)
        with pytest.raises(gpu.NativeError, match="slots"):
            b.add(64, 64)


def test_update_host(gpu, oracle):
    with gpu.BatchedSW(capacity=4) as b:
        ids = [b.add(64, 64, 2.2, 1, (16, 8)), b.add(128, 96, 2.5, 2, (8, 8))]
        ins = [oracle.hot_start(64, 64, 1), oracle.hot_start(128, 96, 1)]
        outs = [np.empty_like(x) for x in ins]
        b.update_host(ids, ins, outs)
    for x, o, (tile, T, seed) in zip(ins, outs, [((16, 8), 2.2, 1), ((8, 8), 2.5, 2)]):
        want, _ = _oracle_run(oracle, x, tile, T, seed, 1)
        assert np.array_equal(o, want)


def test_update_host_contiguous_arena(gpu, oracle):
    """Host buffers that are consecutive slices of one arena (one copy per direction) give the
    same spins as the oracle, for lattices of different sizes; a repeated id is rejected."""
    shapes = [((64, 64), (16, 8), 2.2, 1), ((96, 128), (8, 8), 2.5, 2), ((34, 30), (16, 4), 2.3, 3)]
    with gpu.BatchedSW(capacity=4) as b:
        ids = [b.add(L0, L1, T, seed, tile) for (L0, L1), tile, T, seed in shapes]
        total = sum(L0 * L1 for (L0, L1), _, _, _ in shapes)
        arena_in = gpu.pinned_empty((total,), np.uint8)
        arena_out = gpu.pinned_empty((total,), np.uint8)
        ins, outs, off = [], [], 0
        for (L0, L1), _, _, _ in shapes:
            x = arena_in[off:off + L0 * L1].reshape(L1, L0)
            x[:] = oracle.hot_start(L0, L1, 1)
            ins.append(x)
            outs.append(arena_out[off:off + L0 * L1].reshape(L1, L0))
            off += L0 * L1
        b.update_host(ids, ins, outs)
        for x, o, (_, tile, T, seed) in zip(ins, outs, shapes):
            want, _ = _oracle_run(oracle, np.array(x), tile, T, seed, 1)
            assert np.array_equal(o, want)
        with pytest.raises(gpu.NativeError):
            b.update_host([ids[0], ids[0]], [ins[0], ins[0]], [outs[0], outs[0]])


def test_update_host_sweeps_unlisted_lattices(gpu, oracle):
    """update_host sweeps every lattice once, also those whose spins it does not move."""
    shapes = [((64, 32), (16, 8), 2.2, 5), ((96, 64), (8, 8), 2.4, 6), ((128, 128), (32, 4), 2.3, 7)]
    with gpu.BatchedSW(capacity=4) as b:
        ids, starts = [], []
        for (L0, L1), tile, T, seed in shapes:
            i = b.add(L0, L1, T, seed, tile)
            start = oracle.hot_start(L0, L1, seed)
            b.set_spins(i, start)
            ids.append(i)
            starts.append(start)
        out = np.empty_like(starts[1])
        b.update_host([ids[1]], [starts[1]], [out])
        for i, start, (_, tile, T, seed) in zip(ids, starts, shapes):
            want, _ = _oracle_run(oracle, start, tile, T, seed, 1)
            assert np.array_equal(b.get_spins(i), want)
        want1, _ = _oracle_run(oracle, starts[1], shapes[1][1], shapes[1][2], shapes[1][3], 1)
        assert np.array_equal(out, want1)


def test_host_io_steps(gpu, oracle):
    """HostIO arenas through update_host_io, two steps with swap(): each step's output is the
    oracle's sweep of the previous step's."""
    shapes = [((64, 64), (16, 8), 2.2, 11), ((34, 30), (16, 4), 2.5, 12), ((128, 96), (8, 8), 2.3, 13)]
    with gpu.BatchedSW(capacity=4) as b:
        ids = [b.add(L0, L1, T, seed, tile) for (L0, L1), tile, T, seed in shapes]
        io = b.host_io(ids)
        starts = []
        for x, ((L0, L1), _, _, seed) in zip(io.inputs, shapes):
            x[:] = oracle.hot_start(L0, L1, seed)
            starts.append(np.array(x))
        for _ in range(2):
            b.update_host_io(io)
            io.swap()
        for x, start, (_, tile, T, seed) in zip(io.inputs, starts, shapes):
            want, _ = _oracle_run(oracle, start, tile, T, seed, 2)
            assert np.array_equal(x, want)
        # a lattice added after the plan was made: swept too (unlisted), and the plan is rebuilt
        extra = b.add(32, 32, 2.1, 14, (16, 8))
        start_x = oracle.hot_start(32, 32, 14)
        b.set_spins(extra, start_x)
        b.update_host_io(io)
        io.swap()
        for x, start, (_, tile, T, seed) in zip(io.inputs, starts, shapes):
            want, _ = _oracle_run(oracle, start, tile, T, seed, 3)
            assert np.array_equal(x, want)
        want_x, _ = _oracle_run(oracle, start_x, (16, 8), 2.1, 14, 1)
        assert np.array_equal(b.get_spins(extra), want_x)


def test_assign_instance_follows_the_lattice_set(gpu, oracle):
    """A batch of 16 x 8 / 16 x 4 lattices runs the lean assign instance; adding an 8 x 8 lattice
    switches the round to the all-shapes instance and removing it switches back, and every
    lattice stays on the oracle's sweeps through both changes."""
    shapes = [(128, 64, (16, 8), 2.3, 31), (64, 64, (16, 4), 2.5, 32)]
    with gpu.BatchedSW(capacity=4) as b:
        ids, state = [], []
        for L0, L1, tile, T, seed in shapes:
            i = b.add(L0, L1, T, seed, tile)
            s0 = oracle.hot_start(L0, L1, seed)
            b.set_spins(i, s0)
            ids.append(i)
            state.append([s0.copy(), oracle.rng_init(16, num_tiles(L0, L1, *tile), seed), tile, T])

        def advance(n):
            for st in state:
                for _ in range(n):
                    oracle.sweep(st[0], st[2][0], st[2][1], st[1], T=st[3])

        b.sweep(2)
        advance(2)
        extra = b.add(96, 64, 2.2, 33, (8, 8))
        x0 = oracle.hot_start(96, 64, 33)
        b.set_spins(extra, x0)
        b.sweep(3)
        advance(3)
        want_x, _ = _oracle_run(oracle, x0, (8, 8), 2.2, 33, 3)
        assert np.array_equal(b.get_spins(extra), want_x)
        b.remove(extra)
        b.sweep(2)
        advance(2)
        for i, st in zip(ids, state):
            assert np.array_equal(b.get_spins(i), st[0])


@pytest.mark.parametrize("rounds", [1, 2, 5])
def test_host_io_rounds(gpu, oracle, rounds):
    """update_host_io_rounds: the pipelined rounds through the two HostIO arenas give the
    oracle's sweeps, with the final spins in io.inputs, and lattices not in the HostIO sweep
    once per round too."""
    shapes = [((64, 64), (16, 8), 2.2, 21), ((34, 30), (16, 4), 2.5, 22), ((128, 96), (8, 8), 2.3, 23),
              ((256, 256), (16, 8), 2.27, 24), ((96, 64), (16, 8), 2.4, 25)]
    with gpu.BatchedSW(capacity=8) as b:
        ids = [b.add(L0, L1, T, seed, tile) for (L0, L1), tile, T, seed in shapes]
        extra = b.add(32, 32, 2.1, 26, (16, 8))
        start_x = oracle.hot_start(32, 32, 26)
        b.set_spins(extra, start_x)
        io = b.host_io(ids)
        starts = []
        for x, ((L0, L1), _, _, seed) in zip(io.inputs, shapes):
            x[:] = oracle.hot_start(L0, L1, seed)
            starts.append(np.array(x))
        b.update_host_io_rounds(io, rounds)
        for x, start, (_, tile, T, seed) in zip(io.inputs, starts, shapes):
            want, _ = _oracle_run(oracle, start, tile, T, seed, rounds)
            assert np.array_equal(x, want)
        want_x, _ = _oracle_run(oracle, start_x, (16, 8), 2.1, 26, rounds)
        assert np.array_equal(b.get_spins(extra), want_x)


def test_snapshot_resume_bit_identical(gpu, tmp_path):
    """Preempt a job (snapshot to disk), resume it in another batch and another slot, and in a
    single-lattice handle: every continuation equals the uninterrupted run."""
    from computational_physics_b200 import snapshot
    with gpu.BatchedSW(capacity=4) as b:
        b.add(48, 48, 2.4, 3, (16, 8))
        lid = b.add(96, 64, 2.3, 9, (16, 8))
        b.hot_start(lid, 9)
        b.sweep(7)
        snap = b.snapshot(lid)
        path = str(tmp_path / "job.npz")
        snapshot.save(path, snap)
        b.sweep(5)
        want = b.get_spins(lid)
    loaded = snapshot.load(path)
    assert loaded["sweeps_done"] == 7 and loaded["spins"].shape == (64, 96)
    with gpu.BatchedSW(capacity=4) as b2:
        b2.add(32, 32, 2.0, 1, (16, 8))
        k = b2.add(96, 64, 2.3, 1234, (16, 8))     # other seed: restore replaces the streams
        b2.restore(k, loaded)
        b2.sweep(5)
        assert np.array_equal(b2.get_spins(k), want)
    with gpu.SwendsenWang2D(96, 64, (16, 8), 16, seed_base=77) as sw:
        sw.restore(loaded)
        sw.update(2.3, 5)
        assert np.array_equal(sw.get_spins(), want)
