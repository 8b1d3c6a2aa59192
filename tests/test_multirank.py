"""The multi-process path of bench.py on CPU: world size 2 over gloo, as torchrun starts it.

Ranks share no data (every rank sweeps its own copy of the workload); what they share is the
barrier around the timed region and the max over ranks of the device-measured time.  These
tests run that plumbing with two CPU processes, and the reference arm end to end under torchrun
(rank 0 alone runs the reference CPU path and prints the one JSON line).
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
