"""Serving loop (radik_server_*): a request's result is the same alone, in a
mixed batch stream, in the per-request baseline mode, and from radik_topk --
bit-exact, since the selection is exact and ties go to the lowest positions --
and every request of the mix equals the CPU oracle on its own row."""
import numpy as np
import pytest

import oracle
from radik_b200 import workloads

from conftest import assert_same_selection

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import radik_b200 as rk  # noqa: E402

DEV = "cuda:0"


def _request(n, k, seed, half=False):
    x = workloads.normal(n, seed)
    t = torch.from_numpy(x.astype(np.float16) if half else x).to(DEV)
    return t, torch.empty(k, dtype=t.dtype, device=DEV), torch.empty(k, dtype=torch.int32, device=DEV)


def _mix(count, seed):
    g = workloads.rng(seed)
    ns = g.choice([32000, 128256, 1 << 20, 3 << 20], size=count, p=[0.4, 0.3, 0.2, 0.1])
    ks = g.choice([1, 50, 1024], size=count)
    half = g.random(count) < 0.25
    return [_request(int(n), int(k), 500 + i, bool(h)) for i, (n, k, h) in enumerate(zip(ns, ks, half))]


@pytest.mark.parametrize("sorted_", [True, False])
def test_result_same_alone_and_in_the_mix(sorted_):
    probe = _request(1 << 20, 1024, 7)
    ref_v, ref_i = rk.topk(probe[0], 1024, sorted=sorted_)
    with rk.Server(0, max_n=1 << 22, max_k=1024, slots=3, max_batch_rows=64) as srv:
        srv.submit(probe[0], 1024, probe[1], probe[2], sorted=sorted_)
        srv.drain()
        alone = (probe[1].clone(), probe[2].clone())
        mix = _mix(120, 3)
        outs = []
        for j, (x, v, i) in enumerate(mix):
            srv.submit(x, v.numel(), v, i, sorted=sorted_)
            if j == 60:  # the probe again, in the middle of the stream, fresh buffers
                pv, pi = torch.empty_like(probe[1]), torch.empty_like(probe[2])
                srv.submit(probe[0], 1024, pv, pi, sorted=sorted_)
        srv.drain()
        done = srv.poll(1 << 14)
        assert all(st == 0 for _, st, _ in done)
    key = (lambda v, i: (v, i)) if sorted_ else (lambda v, i: (v[torch.argsort(i)], torch.sort(i)[0]))
    for a, b in ((alone, (pv, pi)), (alone, (ref_v.view(-1), ref_i.view(-1)))):
        ka, kb = key(*a), key(*b)
        assert torch.equal(ka[0], kb[0]) and torch.equal(ka[1], kb[1])
    # every request of the mix against the oracle on its own row
    for j, (x, v, i) in enumerate(mix):
        xh = x.cpu().numpy()
        k = v.numel()
        want = oracle.topk(xh, [xh.size], k, flags=oracle.flags_of(True, sorted_))
        assert_same_selection((v.cpu().numpy(), i.cpu().numpy()), want, [xh.size], [k], [0], sorted_,
                              f"request {j} (n={xh.size}, k={k}, {x.dtype})")


def test_per_request_mode_and_small_budget():
    mix = _mix(40, 11)
    results = []
    for mode, budget in ((1, 0), (0, 64 << 20)):
        outs = [(torch.empty_like(v), torch.empty_like(i)) for _, v, i in mix]
        with rk.Server(0, mode=mode, max_n=1 << 22, max_k=1024, budget_bytes=budget) as srv:
            for (x, v, _), (ov, oi) in zip(mix, outs):
                srv.submit(x, v.numel(), ov, oi, sorted=True)
            srv.drain()
        results.append(outs)
    for (a_v, a_i), (b_v, b_i) in zip(*results):
        assert torch.equal(a_v, b_v) and torch.equal(a_i, b_i)
