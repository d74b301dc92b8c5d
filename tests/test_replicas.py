"""The N > 1 path of bench.py on the CPU: two gloo ranks (127.0.0.1) take the
max of their times and report the whole job's throughput, and the reference
arm under torchrun runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_replicas(world, rank, backend="gloo")
    try:
        t = bench.max_over_ranks(1.5 + rank, dist)  # rank 1 is the slower replica
        out[rank] = (t, bench.whole_job_rate(1000, 10, world, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.5, 1000 * 10 * 2 / 2.5 / 1e6)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_replicas(1, 0) is None
    assert bench.max_over_ranks(3.0, None) == 3.0


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_runs_on_rank_zero_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    if rank == 1:
        assert p.stdout.strip() == ""
    else:
        line = json.loads(p.stdout.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def test_batch_split_is_opt_in(monkeypatch):
    """At N > 1 the default run times replicas only; the split of the 64-case
    batch over the ranks runs only with --batch-split."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2"])
    assert bench.parse().batch_split is False
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2", "--batch-split"])
    assert bench.parse().batch_split is True
