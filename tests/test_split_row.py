"""One row split over several ranks (radik_b200.sharding.split_row_select).

CPU tests run the exchange protocol -- per-level histogram all-reduce, the
identical bin choice on every rank, the gather of selected and tied keys --
over two gloo ranks, with a host stand-in for the two device kernels
(histogram / collect of one shard).  The GPU test runs the same protocol with
the device kernels (radik_shard_histogram / radik_shard_collect) over three
shards of one row on one GPU.  Every result must equal the oracle's selection
of the whole row: values bit-exact, global positions exact (lowest-position
ties)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from radik_b200 import workloads  # noqa: E402
from radik_b200.sharding import _all_gather_cat, _all_reduce_sum, _composites, split_row_select  # noqa: E402

from conftest import bits_of  # noqa: E402


class HostShard:
    """Test stand-in for one rank's device kernels: the same histogram and
    collect on the host, from the same composite order."""

    def __init__(self, x: np.ndarray, pos_base: int, ib: int, largest: bool, with_scale=False, scaler=0.0):
        t = torch.from_numpy(x)
        bits = bits_of(x).astype(np.int64)
        pos = np.arange(pos_base, pos_base + x.size, dtype=np.int64)
        self.entries = torch.from_numpy((bits << 32) | pos)
        self.comp = _composites(self.entries, t.dtype, largest, with_scale, scaler, ib)
        self.w = (32 if (t.dtype == torch.float32 or with_scale) else 16) + ib

    def histogram(self, prefix, plen, d):
        sh = self.w - plen
        m = (self.comp >> sh) == prefix if plen > 0 else torch.ones_like(self.comp, dtype=torch.bool)
        digit = (self.comp[m] >> (sh - d)) & ((1 << d) - 1)
        return torch.bincount(digit, minlength=1 << d).to(torch.int64)

    def collect(self, prefix, plen, cap_b, cap_t):
        t = self.comp >> (self.w - plen) if plen > 0 else torch.zeros_like(self.comp)
        b, ti = self.entries[t < prefix], self.entries[t == prefix]
        return b[:cap_b], ti[:cap_t], b.numel(), ti.numel()


def _row(dist, n, seed, dtype):
    x = {"normal": lambda: workloads.normal(n, seed),
         "ties": lambda: np.floor(workloads.normal(n, seed) * 3).astype(np.float32),
         "zero": lambda: np.zeros(n, np.float32),
         "mantissa": lambda: workloads.mantissa_noise(n, seed)}[dist]()
    return x.astype(np.float16) if dtype == "f16" else x


def _expect(x, k, largest, sorted_):
    v, i = oracle.topk(x, [x.size], k, flags=oracle.flags_of(largest, sorted_))
    return bits_of(v), i.astype(np.int64)


def _check(got, want, sorted_, k, n):
    gv, gi = got
    wv, wi = want
    gb = bits_of(gv.cpu().numpy())
    gi = gi.cpu().numpy()
    m = min(k, n)
    if not sorted_:
        # split-row output is in position order, the oracle's too
        pass
    assert np.array_equal(gi[:m], wi[:m]), "positions differ"
    assert np.array_equal(gb[:m], wv[:m]), "values differ"
    assert np.all(gi[m:] == -1) and np.all(gb[m:] == 0)


@pytest.mark.parametrize("dtype", ["f32", "f16"])
@pytest.mark.parametrize("dist", ["normal", "ties", "zero", "mantissa"])
def test_local_shards_match_oracle(dtype, dist):
    n = 200003
    x = _row(dist, n, 5, dtype)
    cuts = [0, 70001, 70001, 150000, n]  # one empty shard
    for k in (1, 100, 5000):
        for largest, sorted_ in ((True, False), (False, True)):
            from radik_b200.sharding import _finish_split, index_bits
            ib = index_bits(n)
            shards = [HostShard(x[a:b], a, ib, largest) for a, b in zip(cuts[:-1], cuts[1:])]
            got = _finish_split(split_row_select(shards, lambda t: t, lambda t: t, n, k, torch.from_numpy(x).dtype,
                                                 largest, sorted=sorted_, cap=2048), k,
                                torch.from_numpy(x).dtype, "cpu")
            _check(got, _expect(x, k, largest, sorted_), sorted_, k, n)


def test_k_above_row_length_idle_fills():
    from radik_b200.sharding import _finish_split, index_bits

    x = workloads.normal(50, 3)
    ib = index_bits(50)
    shards = [HostShard(x[:20], 0, ib, True), HostShard(x[20:], 20, ib, True)]
    got = _finish_split(split_row_select(shards, lambda t: t, lambda t: t, 50, 64, torch.float32, True, sorted=True),
                        64, torch.float32, "cpu")
    _check(got, _expect(x, 64, True, True), True, 64, 50)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from radik_b200.sharding import _finish_split, index_bits

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ok = True
    try:
        n = 300007
        for dist_name, k, largest, sorted_ in (("normal", 256, True, False), ("ties", 4000, False, True),
                                               ("zero", 77, True, True), ("mantissa", 1, True, False)):
            x = _row(dist_name, n, 9, "f32")
            cut = [0, 123457, n]
            a, b = cut[rank], cut[rank + 1]
            ib = index_bits(n)
            shard = HostShard(x[a:b], a, ib, largest)
            got = _finish_split(split_row_select([shard], lambda t: _all_reduce_sum(t, None),
                                                 lambda t: _all_gather_cat(t, None), n, k, torch.float32, largest,
                                                 sorted=sorted_, cap=1024), k, torch.float32, "cpu")
            want = _expect(x, k, largest, sorted_)
            try:
                _check(got, want, sorted_, k, n)
            except AssertionError:
                ok = False
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_select_the_single_row_result():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: True, 1: True}


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f32", "f16"])
@pytest.mark.parametrize("dist", ["normal", "ties", "mantissa"])
def test_device_shards_match_oracle(dtype, dist):
    """The device kernels behind the protocol: three shards of one 2^22-key
    row on one GPU (the exchanges are local sums)."""
    from radik_b200.sharding import topk_split_row_local

    n = (1 << 22) + 13
    x = _row(dist, n, 21, dtype)
    cuts = [0, 1 << 20, 3 << 20, n]
    t = torch.from_numpy(x).to("cuda:0")
    shards = [t[a:b] for a, b in zip(cuts[:-1], cuts[1:])]
    for k in (16, 1024, 20000):
        for largest, sorted_ in ((True, False), (False, True)):
            got = topk_split_row_local(shards, k, pos_bases=cuts[:-1], n_total=n, largest=largest, sorted=sorted_)
            _check(got, _expect(x, k, largest, sorted_), sorted_, k, n)
