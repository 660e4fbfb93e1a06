"""Multi-rank host logic of the batched path, on CPU: the problem list is
shared out over ranks by cell count with no data-path exchange, every rank
derives the same assignment on its own, and the step time reported is the max
over ranks.  The two-rank case runs as real processes over gloo."""
import os
import socket

import numpy as np
import pytest

from dspw import workloads as W
from dspw.partition import imbalance, loads, partition


def test_partition_covers_each_problem_once():
    rng = np.random.default_rng(0)
    cells = rng.integers(1, 10_000, 500).tolist()
    for world in (1, 2, 3, 8):
        parts = partition(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        assert sum(loads(cells, parts)) == sum(cells)
        # greedy largest-first: no rank exceeds the mean by more than the largest problem
        assert max(loads(cells, parts)) <= sum(cells) / world + max(cells)


def test_partition_is_deterministic_and_balanced_for_the_batch():
    cells = [W.spec_cells(s) for s in W.batched_specs()]
    assert partition(cells, 4) == partition(list(cells), 4)
    assert imbalance(cells, partition(cells, 2)) < 1.01
    # one 2048^2 vortex level holds a quarter of all cells: it bounds 8-way balance
    assert max(cells) == 2048 * 2048
    assert imbalance(cells, partition(cells, 8)) == pytest.approx(max(cells) / (sum(cells) / 8))


def test_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5], 2) == [[0], []]
    with pytest.raises(ValueError):
        partition([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        specs = W.batched_specs(levels=(16, 32, 64), nburgers=40, burgers_nx=(100, 400), seed=5)
        cells = [W.spec_cells(s) for s in specs]
        mine = partition(cells, world)[rank]
        descs, prims, ncell = W.batched("fp64", "sp_weno", None, levels=(16, 32, 64), nburgers=40,
                                        burgers_nx=(100, 400), seed=5, select=mine)
        assert len(descs) == len(mine) and ncell == sum(cells[i] for i in mine)
        # every rank's view of the assignment
        got = [None] * world
        dist.all_gather_object(got, mine)
        # the timing reduction of the bench: max over ranks of the device time
        t = torch.tensor([10.0 + rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = torch.tensor([float(ncell)], dtype=torch.float64)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        q.put((rank, got, float(t.item()), float(tot.item()), sum(cells)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    views = [r[1] for r in res]
    assert views[0] == views[1]
    a, b = views[0]
    assert not set(a) & set(b) and sorted(a + b) == list(range(len(a) + len(b)))
    for _, _, tmax, tot, total_cells in res:
        assert tmax == 11.0
        assert tot == total_cells
