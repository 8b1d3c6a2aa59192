"""The multi-process path of bench.py on CPU: world size 2 over gloo, as torchrun starts it.

Ranks share no data on the data path: the batched mix and the serving queue are sharded (every
lattice or job on one rank), and what travels is the barrier around the timed region, the max
over ranks of the device-measured time and the per-lattice results gathered on rank 0.  These
tests run that plumbing with two CPU processes (the C restatement of the sweep stands in for the
GPU engine), and the reference arm end to end under torchrun (rank 0 alone runs the reference
CPU path and prints the one JSON line).
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    m = d.max(1.5 + rank)          # each rank's "device time"; every rank must see the max
    d.barrier()
    d.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"world": d.world, "rank": d.rank, "max": m}, f)


def test_dist_barrier_and_max_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [g["rank"] for g in got] == [0, 1]
    assert all(g["world"] == 2 and g["max"] == 2.5 for g in got)


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload", "plain1024"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=540, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["n_gpus"] == 2 and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"


# A small mix for the sharded run: (L, T, seed); the C restatement sweeps each lattice.
SMALL_MIX = [(L, T, 100 + k) for k, (L, T) in enumerate(
    [(16, 2.0), (32, 2.3), (48, 2.6), (64, 2.2), (16, 2.5), (32, 2.1), (64, 2.4), (48, 2.0), (32, 2.6), (16, 2.2),
     (64, 2.0), (48, 2.3)])]


def _small_mix_results(indices) -> dict:
    """{mix index: [e, m, lcg32 iteration sum]} after hot start + 3 sweeps (tile 16 x 8, W 16)."""
    from oracle import Oracle, num_tiles
    o = Oracle()
    out = {}
    for k in indices:
        L, T, seed = SMALL_MIX[k]
        spins = o.hot_start(L, L, seed)
        rng = o.rng_init(16, num_tiles(L, L, 16, 8), seed)
        for _ in range(3):
            o.sweep(spins, 16, 8, rng, T=T)
        e, m = o.energy_magnetization(spins)
        out[k] = [int(e), int(m), int(rng.iteration.sum())]
    return out


def _shard_rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    from computational_physics_b200 import shard
    d = bench.Dist()
    weights = [shard.lattice_bytes(L, L, (16, 8)) for L, _, _ in SMALL_MIX]
    mine = shard.shard_of(weights, world, rank)
    merged = shard.gather_results(_small_mix_results(mine), d.gather_object)
    d.barrier()
    d.close()
    with open(os.path.join(out_dir, f"shard{rank}.json"), "w") as f:
        json.dump({"mine": mine, "merged": merged}, f)


def test_sharded_mix_gathers_the_one_rank_results(tmp_path):
    """Two ranks sweep disjoint halves of a mix; rank 0's gathered per-lattice results equal a
    one-process run over the whole mix, every lattice is reported once."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_shard_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [json.load(open(tmp_path / f"shard{r}.json")) for r in range(2)]
    mine = [set(g["mine"]) for g in got]
    assert mine[0].isdisjoint(mine[1]) and mine[0] | mine[1] == set(range(len(SMALL_MIX)))
    assert got[1]["merged"] is None
    merged = {int(k): v for k, v in got[0]["merged"].items()}
    assert merged == _small_mix_results(range(len(SMALL_MIX)))


@pytest.mark.parametrize("world", [2, 4, 8])
def test_bench_mix_partition_is_balanced(world):
    """The 512-lattice mix over `world` ranks: each lattice on exactly one rank, device bytes
    within 10 % of the mean on every rank."""
    sys.path.insert(0, ROOT)
    import bench
    parts, imbalance = bench.mix_shards(world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(bench.mix_workload())))
    assert imbalance <= 1.10, imbalance
