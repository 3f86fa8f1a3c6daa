"""Rows across ranks (CPU, gloo, world size 2): contiguous Sigma-n balanced
ranges, each rank selecting its own rows (here with the CPU oracle, the GPU
library's checker), and an all_gather that reassembles the single-process
result exactly."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from radik_b200 import workloads  # noqa: E402
from radik_b200.sharding import shard_bounds, shard_rows  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ranges_cover_rows_in_order_and_balance(world):
    ns, _ = workloads.uneven_rows(200, 4, 10, 20, 64)
    b = shard_bounds(ns, world)
    assert b[0][0] == 0 and b[-1][1] == len(ns)
    assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
    assert all(hi > lo for lo, hi in b)
    sums = [sum(ns[lo:hi]) for lo, hi in b]
    assert max(sums) - min(sums) <= 2 * max(ns)


def test_fewer_rows_than_ranks():
    b = shard_bounds([5, 7], 4)
    assert b[0][0] == 0 and b[-1][1] == 2 and sum(hi - lo for lo, hi in b) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from radik_b200.sharding import gather_rows

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        B, n, k = 24, 5000, 37
        x = np.concatenate([workloads.normal(n, 60 + r) for r in range(B)])
        lo, hi = shard_rows([n] * B, world, rank)
        v, i = oracle.topk(x[lo * n:hi * n], [n] * (hi - lo), k, flags=oracle.flags_of(True, True))
        gv, gi = gather_rows(torch.from_numpy(v.reshape(hi - lo, k)), torch.from_numpy(i.reshape(hi - lo, k)), k,
                             [n] * B)
        if rank == 0:
            fv, fi = oracle.topk(x, [n] * B, k, flags=oracle.flags_of(True, True))
            q.put(bool(np.array_equal(gv.numpy().reshape(-1), fv) and np.array_equal(gi.numpy().reshape(-1), fi)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_the_single_process_result():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) is True
