"""Instance sharding for the multi-GPU batched / served modes, exercised on CPU: the split
covers every instance once and balances the work, and the gather / max-over-ranks
collectives assemble the same result as one process, with world size 2 over gloo."""
import os
import socket

import numpy as np
import pytest

from hphi_b200 import shard

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    dims = rng.choice([48620, 184756, 705432, 2704156], size=256)
    for world in (1, 2, 3, 8):
        parts = shard.partition(dims, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(dims)))
        loads = [sum(int(dims[i]) for i in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest item
        assert max(loads) - sum(loads) / world <= max(dims)
    assert shard.partition([5, 3], 4)[2:] == [[], []]


def test_gather_single_process():
    vals = np.array([[1.0, 2.0], [3.0, 4.0]])
    out = shard.gather(vals, [2, 0], 3)
    assert np.array_equal(out, [[3.0, 4.0], [0.0, 0.0], [1.0, 2.0]])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, dims, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parts = shard.partition(dims, world)
        mine = parts[rank]
        # stand-in for each instance's results: (energy, steps) computed from its index
        vals = np.array([[-float(i) * 0.5, 10.0 + i] for i in mine]).reshape(len(mine), 2)
        out = shard.gather(vals, mine, len(dims), dist)
        t = shard.max_over_ranks(1.0 + rank, dist)
        q.put((rank, out.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
    dims = [7, 3, 9, 1, 4, 4]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, dims, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [[-i * 0.5, 10.0 + i] for i in range(len(dims))]
    for rank, out, t in res:
        assert out == expect
        assert t == 2.0
