"""Multi-rank placement of complexes (CPU, gloo, world size 2).

The docking path shards by complex with no collective on its data; the
ranks only reduce the slowest device time and the work counters.  These
tests run the real torch.distributed plumbing on CPU processes."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gpudock_b200 import shard


def test_place_is_a_balanced_partition():
    rng = np.random.default_rng(0)
    costs = [shard.complex_cost(32, int(n), 6000) for n in rng.integers(12, 97, 512)]
    for ws in (1, 2, 3, 8):
        parts = shard.place(costs, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT: no rank exceeds the mean by more than the largest single cost
        assert max(loads) - sum(loads) / ws <= max(costs) + 1e-6
    assert shard.place([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.place([1.0], 0)
    with pytest.raises(ValueError):
        shard.my_items([1.0], 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, costs, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.my_items(costs, ws, rank)
        work = sum(costs[i] for i in mine)
        slowest = shard.max_over_ranks(1.0 + rank)  # per-rank "device time"
        total = shard.sum_over_ranks(work)
        lists = [None] * ws
        dist.all_gather_object(lists, mine)
        out[rank] = (lists, slowest, total)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ws = 2
    costs = [float(c) for c in np.random.default_rng(1).integers(1, 100, 37)]
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, costs, out)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(ws):
        lists, slowest, total = out[r]
        assert sorted(i for l in lists for i in l) == list(range(len(costs)))
        assert not set(lists[0]) & set(lists[1])
        assert slowest == 2.0
        assert total == pytest.approx(sum(costs))
