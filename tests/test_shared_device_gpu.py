"""radik_topk_rows_ctas: the rows form on part of the device.

The engine runs one CTA per SM; with max_ctas it takes fewer SMs, in a
launch that is not cooperative, so calls on other streams can run beside it
(the serving loop admits batches this way).  Every grid size must select exactly as the
whole device does: each case is checked against the CPU oracle, including
grids of one and a few CTAs, radix rows, rows that fall back to the grid-wide
tail (all keys tied) and two calls in flight at once on disjoint SMs."""
import numpy as np
import pytest

import oracle
from radik_b200 import workloads

from conftest import assert_same_selection

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import radik_b200 as rk  # noqa: E402

DEV = "cuda:0"


def _rows_case(ns, ks, seed, dist="normal"):
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int64)
    if dist == "normal":
        x = workloads.normal(int(sum(ns)), seed)
    else:  # every key tied: the selection comes down to positions
        x = np.full(int(sum(ns)), 0.5, np.float32)
    rows = [(int(a), int(b), int(n), int(k)) for a, b, n, k in zip(offs, oo, ns, ks)]
    return x, rows, [int(v) for v in oo]


def _check(x, rows, oo, got, sorted_, label):
    ns = [r[2] for r in rows]
    ks = [r[3] for r in rows]
    want = oracle.topk(x, ns, ks, flags=oracle.flags_of(True, sorted_), out_offsets=oo)
    assert_same_selection((got[0].cpu().numpy(), got[1].cpu().numpy()), want, ns, ks, oo, sorted_, label)


CASES = {
    "mixed": ([1000, 40000, 300000, 1 << 20, 5000, 2 << 20], [10, 256, 1000, 256, 5000, 2048]),
    "radix": ([1 << 18, 100000], [20000, 6000]),
    "many_small": ([32000] * 64, [50] * 64),
}


@pytest.mark.parametrize("ctas", [1, 3, 37, 111])
@pytest.mark.parametrize("case", sorted(CASES))
def test_small_grids_select_exactly(case, ctas):
    ns, ks = CASES[case]
    x, rows, oo = _rows_case(ns, ks, 40 + ctas)
    t = torch.from_numpy(x).to(DEV)
    for sorted_ in (False, True):
        got = rk.topk_rows(t, rows, sorted=sorted_, max_ctas=ctas)
        _check(x, rows, oo, got, sorted_, f"{case} ctas={ctas} sorted={sorted_}")


@pytest.mark.parametrize("ctas", [2, 16])
def test_tied_rows_on_small_grids(ctas):
    # all keys equal: the candidate sets overflow and the grid-wide tail runs
    x, rows, oo = _rows_case([1 << 20, 300000], [4096, 100], 0, dist="tied")
    t = torch.from_numpy(x).to(DEV)
    got = rk.topk_rows(t, rows, max_ctas=ctas)
    _check(x, rows, oo, got, False, f"tied ctas={ctas}")


def test_two_calls_side_by_side_on_disjoint_sms():
    total = rk.engine_ctas()
    a_ctas = total * 3 // 4
    b_ctas = total - a_ctas
    xa, rows_a, oo_a = _rows_case([1 << 22, 1 << 21], [256, 1024], 71)
    xb, rows_b, oo_b = _rows_case([32000] * 48 + [128256] * 16, [50] * 48 + [1024] * 16, 72)
    ta, tb = torch.from_numpy(xa).to(DEV), torch.from_numpy(xb).to(DEV)
    sa, sb = torch.cuda.Stream(DEV), torch.cuda.Stream(DEV)
    torch.cuda.synchronize()
    for _ in range(3):
        # each call's descriptors, workspace and outputs are allocated on its
        # own stream, so the caching allocator never hands one call's memory
        # to the other while it runs
        with torch.cuda.stream(sa):
            ga = rk.topk_rows(ta, rows_a, max_ctas=a_ctas, check=False)
        with torch.cuda.stream(sb):
            gb = rk.topk_rows(tb, rows_b, max_ctas=b_ctas, check=False)
        torch.cuda.synchronize()
        _check(xa, rows_a, oo_a, ga, False, "side by side, large batch")
        _check(xb, rows_b, oo_b, gb, False, "side by side, small batch")


def test_max_ctas_is_validated():
    x = torch.zeros(1000, device=DEV)
    with pytest.raises(rk.RadikError) as err:
        rk.topk_rows(x, [(0, 0, 1000, 10)], max_ctas=-1)
    assert err.value.code == rk.EINVAL


def test_server_runs_batches_beside_each_other():
    g = workloads.rng(5)
    reqs = []
    for j in range(60):
        n = int(g.choice([32000, 128256, 1 << 20, 1 << 22], p=[0.4, 0.3, 0.2, 0.1]))
        k = int(g.choice([1, 50, 1024]))
        x = torch.from_numpy(workloads.normal(n, 900 + j)).to(DEV)
        reqs.append((x, torch.empty(k, device=DEV), torch.empty(k, dtype=torch.int32, device=DEV)))
    with rk.Server(0, max_n=1 << 22, max_k=1024, slots=3, max_batch_rows=8) as srv:
        for x, v, i in reqs:
            srv.submit(x, v.numel(), v, i)
        srv.drain()
        st = srv.stats()
    assert st["batches"] >= 8 and st["requests"] == len(reqs)
    assert st["ctas_total"] == rk.engine_ctas() and st["ctas_cap"] == st["ctas_total"] * 3 // 4
    assert st["max_ctas_in_flight"] <= st["ctas_total"]
    # with 60 requests queued at once, later batches start while earlier ones run
    assert st["batches_beside_others"] > 0 and st["max_batches_in_flight"] >= 2
    for j, (x, v, i) in enumerate(reqs):
        xh = x.cpu().numpy()
        want = oracle.topk(xh, [xh.size], v.numel(), flags=oracle.flags_of(True, False))
        assert_same_selection((v.cpu().numpy(), i.cpu().numpy()), want, [xh.size], [v.numel()], [0], False,
                              f"request {j}")


def test_call_span_is_recorded():
    x, rows, oo = _rows_case([1 << 20, 40000], [256, 64], 7)
    t = torch.from_numpy(x).to(DEV)
    flags = rk.make_flags(True, False)
    ws = torch.empty(rk.get_rows_workspace_size(rk.F32, len(rows), sum(r[2] for r in rows), 1 << 20, 256, flags),
                     dtype=torch.uint8, device=DEV)
    got = rk.topk_rows(t, rows, workspace=ws, max_ctas=20)
    t0, t1 = rk.call_span(ws)
    assert 0 < t0 < t1 and t1 - t0 < 10**9  # nanoseconds of the GPU global timer
    _check(x, rows, oo, got, False, "span call")
