"""Case distribution over ranks (aerocfd_b200/distribute.py), on the CPU: the
longest-processing-time split covers every case once and stays within
Graham's bound, and two gloo ranks, each iterating its share of a case list
through the oracle, gather the same per-case results as one process running
the whole list."""
import os
import socket

import numpy as np
import pytest

from aerocfd_b200 import distribute, grids


def test_assign_covers_every_case_once_and_balances():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        for n in (0, 1, 5, 64):
            costs = rng.integers(1_000, 100_000, size=n)
            parts = distribute.assign(costs, world)
            assert len(parts) == world
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            assert distribute.assign(costs, world) == parts      # the same on every rank
            if n:
                loads = [int(sum(costs[p])) for p in parts]
                lower = max(costs.sum() / world, costs.max())
                assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
    with pytest.raises(ValueError):
        distribute.assign([1, 2], 0)


def test_assign_uneven_batch_of_the_bench():
    cases = grids.bump_batch(64, seed=0)
    nodes = [c.nodes for c in cases]
    for world in (2, 4, 8):
        parts = distribute.assign(nodes, world)
        loads = [sum(nodes[i] for i in p) for p in parts]
        assert max(loads) / (sum(nodes) / world) < 1.05, (world, loads)


def small_cases():
    return [grids.bump_channel(ni=17 + 4 * i, nj=9, nk=3) for i in range(5)]


def run_cases(indices, cases, oracle_mod):
    out = {}
    for i, c in zip(indices, cases):
        oc = oracle_mod.OracleCase(c, fast=True)
        oc.geometry()
        oc.init_flowfield()
        oc.start()
        out[i] = oc.iterate(3)
    return out


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import oracle as oracle_mod
        cases = small_cases()
        idx, mine = distribute.share(cases, rank, world)
        res = distribute.gather(run_cases(idx, mine, oracle_mod), dist)
        if rank == 0:
            q.put({k: v.tolist() for k, v in res.items()})
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_single_process_results(oracle_mod):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    got = q.get()
    cases = small_cases()
    want = run_cases(range(len(cases)), cases, oracle_mod)
    assert sorted(got) == list(range(len(cases)))
    for i in want:
        assert np.array_equal(np.array(got[i]), want[i]), i
