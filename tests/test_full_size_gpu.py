"""GPU parity at the benchmark's own sizes, and on IEEE edge values.

Every configuration the throughput figures are quoted on is checked here at
its real size: the CUDA library against the CPU oracle (values bit-exact,
index sets exact, lowest-position ties) and, where the reference RadiK can run
the same call, against RadiK's value multisets (its own check compares values
only: radik/test/test_radik.cu:188-213).  All calls go through the C ABI.
"""
import numpy as np
import pytest

import oracle
from radik_b200 import workloads

from conftest import assert_same_selection, bits_of

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import radik_b200 as rk  # noqa: E402

DEV = "cuda:0"
B256, N20 = 256, 1 << 20


@pytest.fixture(scope="module")
def rows256():
    """The batched benchmark input: 256 rows of U(0,1), row r from seed r."""
    x = workloads.uniform_rows(B256, N20, 0)
    return x, torch.from_numpy(x.reshape(-1)).to(DEV)


@pytest.fixture(scope="module")
def ref():
    try:
        return oracle.RefRadik()
    except FileNotFoundError as e:
        pytest.skip(str(e))


def _gpu(t, B, k, sorted_, largest, ascend=None):
    gv, gi = rk.topk(t, k, [t.numel() // B] * B, largest=largest, sorted=sorted_, ascend=ascend)
    return gv.cpu().numpy().reshape(-1), gi.cpu().numpy().reshape(-1)


def _ref_values(ref, t, B, n, k, largest, ascend, sorted_):
    dt = rk.F16 if t.dtype == torch.float16 else rk.F32
    vo = torch.zeros(B * k, dtype=t.dtype, device=DEV)
    io = torch.zeros(B * k, dtype=torch.int32, device=DEV)
    ws = torch.zeros(ref.workspace_size(dt, k, n, B), dtype=torch.uint8, device=DEV)
    ref.topk(dt, largest, ascend, False, sorted_, t.data_ptr(), vo.data_ptr(), io.data_ptr(), ws.data_ptr(),
             [n] * B, k, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return bits_of(vo.cpu().numpy()).reshape(B, k), io.cpu().numpy().reshape(B, k).astype(np.int64)


# ---------------------------------------------------------------------------
# 256 x 2^20: every batched configuration of the benchmark
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("k", [32, 256, 1024])
@pytest.mark.parametrize("sorted_", [False, True], ids=["unsorted", "sorted"])
def test_batched_256x1M_f32(rows256, k, sorted_):
    x, t = rows256
    got = _gpu(t, B256, k, sorted_, True)
    want = oracle.topk(x.reshape(-1), [N20] * B256, k, flags=oracle.flags_of(True, sorted_))
    assert_same_selection(got, want, [N20] * B256, [k] * B256, [r * k for r in range(B256)], sorted_, f"k={k}")


def test_batched_256x1M_f16_k256(rows256):
    x, _ = rows256
    xh = x.astype(np.float16)
    t = torch.from_numpy(xh.reshape(-1)).to(DEV)
    for sorted_ in (False, True):
        got = _gpu(t, B256, 256, sorted_, True)
        want = oracle.topk(xh.reshape(-1), [N20] * B256, 256, flags=oracle.flags_of(True, sorted_))
        assert_same_selection(got, want, [N20] * B256, [256] * B256, [r * 256 for r in range(B256)], sorted_, "f16")


def test_batched_256x1M_smallest_ascending(rows256):
    """The reference driver's default mode: smallest-k, ascending, sorted
    (radik/test/test_radik.cu:18-19)."""
    x, t = rows256
    got = _gpu(t, B256, 256, True, False, ascend=True)
    want = oracle.topk(x.reshape(-1), [N20] * B256, 256, flags=oracle.flags_of(False, True, True))
    assert_same_selection(got, want, [N20] * B256, [256] * B256, [r * 256 for r in range(B256)], True, "smallest")


@pytest.mark.parametrize("case", [(256, True, False, False), (32, True, False, True), (1024, False, True, True)],
                         ids=["k256-largest", "k32-largest-sorted", "k1024-smallest-asc"])
def test_batched_256x1M_value_multisets_match_reference(rows256, ref, case):
    k, largest, ascend, sorted_ = case
    x, t = rows256
    rv, ri = _ref_values(ref, t, B256, N20, k, largest, ascend, sorted_)
    gv, _ = rk.topk(t, k, [N20] * B256, largest=largest, sorted=sorted_, ascend=ascend)
    gv = bits_of(gv.cpu().numpy()).reshape(B256, k)
    assert np.array_equal(np.sort(rv, 1), np.sort(gv, 1))
    if sorted_:
        assert np.array_equal(rv, gv)
    # RadiK's indices are a valid selection of its own values
    rows = bits_of(x).reshape(B256, N20)
    assert np.array_equal(np.take_along_axis(rows, ri, 1), rv)


def test_batched_256x1M_f16_value_multisets_match_reference(rows256, ref):
    x, _ = rows256
    t = torch.from_numpy(x.astype(np.float16).reshape(-1)).to(DEV)
    rv, _ = _ref_values(ref, t, B256, N20, 256, True, False, True)
    gv, _ = rk.topk(t, 256, [N20] * B256, largest=True, sorted=True)
    assert np.array_equal(rv, bits_of(gv.cpu().numpy()).reshape(B256, 256))


# ---------------------------------------------------------------------------
# S1: the single-row configuration
# ---------------------------------------------------------------------------
def test_single_row_S1_against_oracle_and_reference(ref):
    x = workloads.uniform01(N20, 0)
    t = torch.from_numpy(x).to(DEV)
    got = _gpu(t, 1, 256, False, True)
    want = oracle.topk(x, [N20], 256, flags=oracle.flags_of(True, False))
    assert_same_selection(got, want, [N20], [256], [0], False, "S1")
    rv, ri = _ref_values(ref, t, 1, N20, 256, True, False, False)
    assert np.array_equal(np.sort(rv[0]), np.sort(bits_of(got[0])))
    assert np.array_equal(bits_of(x)[ri[0]], rv[0]) and len(np.unique(ri[0])) == 256


# ---------------------------------------------------------------------------
# Skew sweep: all 52 cases (n = 2^24, k = 2^4..2^16, four distributions)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dist", list(workloads.SKEW_DISTRIBUTIONS))
def test_skew_sweep_all_cases(dist):
    """Every case of the sweep, largest-k unsorted as benchmarked: the top-k
    for every k is the prefix of the row's sorted top-65536 (composite order:
    key, then lowest position), so one oracle call covers the 13 cases."""
    n = 1 << 24
    x = workloads.skew_row(dist, n, 11)
    t = torch.from_numpy(x).to(DEV)
    ov, oi = oracle.topk(x, [n], 1 << 16, flags=oracle.flags_of(True, True))
    ov, oi = bits_of(ov), oi.astype(np.int64)
    ws = torch.empty(rk.get_radix_select_l_workspace_size(rk.F32, 1 << 16, n, 1, 0), dtype=torch.uint8, device=DEV)
    for e in range(4, 17):
        k = 1 << e
        gv, gi = rk.topk(t, k, [n], largest=True, sorted=False, workspace=ws)
        gv, gi = bits_of(gv.cpu().numpy().reshape(-1)), gi.cpu().numpy().reshape(-1).astype(np.int64)
        o, w = np.argsort(gi), np.argsort(oi[:k])
        assert np.array_equal(gi[o], oi[:k][w]), f"{dist} k={k}: index sets differ"
        assert np.array_equal(gv[o], ov[:k][w]), f"{dist} k={k}: values differ"


# ---------------------------------------------------------------------------
# Uneven batch: the benchmark's exact 4096-row set
# ---------------------------------------------------------------------------
def test_uneven_4096_rows_as_benchmarked():
    B = 4096
    ns, ks = workloads.uneven_rows(B, 7)
    total_n = sum(ns)
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int64)
    x = workloads.uneven_device_values(total_n, 7, torch.device(DEV))
    rows = [(int(a), int(b), int(n), int(k)) for a, b, n, k in zip(offs, oo, ns, ks)]
    gv, gi = rk.topk_rows(x, rows, largest=True, sorted=False)
    xh = x.cpu().numpy()
    del x
    ov, oi = oracle.topk(xh, ns, ks, flags=oracle.flags_of(True, False), out_offsets=[int(v) for v in oo])
    assert_same_selection((gv.cpu().numpy(), gi.cpu().numpy()), (ov, oi), ns, ks, oo, False, "uneven 4096")


def test_uneven_device_values_are_reproducible():
    a = workloads.uneven_device_values(3 << 20, 7, torch.device(DEV))
    b = workloads.uneven_device_values(3 << 20, 7, torch.device(DEV))
    assert torch.equal(a, b)
    assert abs(float(a.mean())) < 0.01 and abs(float(a.std()) - 1.0) < 0.01


# ---------------------------------------------------------------------------
# NaN, +-0 and +-inf
# ---------------------------------------------------------------------------
F32_SPECIAL = np.array([0x7FC00000, 0x7F800001, 0x7FFFFFFF, 0xFFC00000, 0xFF800001, 0x7F800000, 0xFF800000,
                        0x00000000, 0x80000000, 0x00000001, 0x80000001], dtype=np.uint32)
F16_SPECIAL = np.array([0x7E00, 0x7C01, 0x7FFF, 0xFE00, 0x7C00, 0xFC00, 0x0000, 0x8000, 0x0001, 0x8001],
                       dtype=np.uint16)
BF16_SPECIAL = np.array([0x7FC0, 0x7F81, 0x7FFF, 0xFFC0, 0x7F80, 0xFF80, 0x0000, 0x8000, 0x0001, 0x8001],
                        dtype=np.uint16)


def edge_row(n, seed, dtype, frac):
    """N(0,1) values with a fraction `frac` of the positions replaced by NaNs
    of several payloads and signs, +-inf, +-0 and +-denormal minima."""
    g = workloads.rng(seed)
    x = workloads.normal(n, seed)
    if dtype == rk.F16:
        b = x.astype(np.float16).view(np.uint16).copy()
        sp = F16_SPECIAL
    elif dtype == rk.BF16:
        b = workloads.to_bf16_bits(x).copy()
        sp = BF16_SPECIAL
    else:
        b = x.view(np.uint32).copy()
        sp = F32_SPECIAL
    pos = g.random(n) < frac
    b[pos] = sp[g.integers(0, len(sp), int(pos.sum()))]
    return b.view(np.float16) if dtype == rk.F16 else b if dtype == rk.BF16 else b.view(np.float32)


def _to_dev(flat, dtype):
    t = torch.from_numpy(np.ascontiguousarray(flat))
    return (t.view(torch.bfloat16) if dtype == rk.BF16 else t).to(DEV)


def _host_values(gv, dtype):
    gv = gv.view(torch.int16) if dtype == rk.BF16 else gv
    v = gv.cpu().numpy().reshape(-1)
    return v.view(np.uint16) if dtype == rk.BF16 else v


@pytest.mark.parametrize("dtype", [rk.F32, rk.F16, rk.BF16], ids=["f32", "f16", "bf16"])
@pytest.mark.parametrize("B,n,k", [(1, 100000, 300), (4, 1 << 20, 256), (1, 1 << 20, 20000), (1, 1 << 22, 4096),
                                   (3, 5000, 77)])
@pytest.mark.parametrize("frac", [0.002, 0.3])
def test_nan_zero_inf_rows_match_oracle(dtype, B, n, k, frac):
    """The oracle's rule, which the library follows: keys are the
    order-preserving integers of the bit patterns, so -0 ranks below +0, a
    positive NaN ranks above +inf by its payload and a negative NaN below
    -inf.  (RadiK instead skips NaN in its first histogram and compares
    floats in its filter: radik/RadixSelect/radixselect_l.cuh:189-194.)"""
    flat = np.concatenate([edge_row(n, 300 + r, dtype, frac) for r in range(B)])
    t = _to_dev(flat, dtype)
    for largest, sorted_ in ((True, False), (False, True), (True, True)):
        gv, gi = rk.topk(t, k, [n] * B, largest=largest, sorted=sorted_)
        want = oracle.topk(flat, [n] * B, k, flags=oracle.flags_of(largest, sorted_), dtype=dtype)
        assert_same_selection((_host_values(gv, dtype), gi.cpu().numpy().reshape(-1)), want, [n] * B, [k] * B,
                              [r * k for r in range(B)], sorted_, f"largest={largest} sorted={sorted_}")


@pytest.mark.parametrize("dtype", [rk.F32, rk.F16, rk.BF16], ids=["f32", "f16", "bf16"])
@pytest.mark.parametrize("largest", [True, False])
def test_signed_zero_rows(dtype, largest):
    """Rows of +-0 (with a few +-1 for the 16-bit hit path): the threshold
    lands on a zero, where float compares do not give the key order."""
    n = 300000
    g = workloads.rng(5)
    x = np.where(g.random(n) < 0.5, np.float32(0.0), np.float32(-0.0)).astype(np.float32)
    u = g.random(n)
    x[u < 0.0005] = 1.0
    x[(u >= 0.0005) & (u < 0.001)] = -1.0
    flat = x.astype(np.float16) if dtype == rk.F16 else workloads.to_bf16_bits(x) if dtype == rk.BF16 else x
    t = _to_dev(flat, dtype)
    gv, gi = rk.topk(t, 1000, [n], largest=largest, sorted=True)
    want = oracle.topk(flat, [n], 1000, flags=oracle.flags_of(largest, True), dtype=dtype)
    assert_same_selection((_host_values(gv, dtype), gi.cpu().numpy().reshape(-1)), want, [n], [1000], [0], True)


@pytest.mark.parametrize("B,n,k", [(4, 1 << 20, 256), (1, 1 << 22, 4096), (8, 200000, 1000)])
def test_inf_rows_value_multisets_match_reference(ref, B, n, k):
    """Rows of finite values with +-inf mixed in (no NaN, no zeros): RadiK's
    value multisets equal ours."""
    rows = []
    for r in range(B):
        g = workloads.rng(600 + r)
        x = workloads.normal(n, 600 + r)
        x[x == 0] = np.float32(1e-3)
        m = g.random(n)
        x[m < 0.0001] = np.inf
        x[(m >= 0.0001) & (m < 0.0002)] = -np.inf
        rows.append(x)
    flat = np.concatenate(rows)
    t = torch.from_numpy(flat).to(DEV)
    for largest in (True, False):
        rv, _ = _ref_values(ref, t, B, n, k, largest, not largest, True)
        gv, _ = rk.topk(t, k, [n] * B, largest=largest, sorted=True)
        assert np.array_equal(rv, bits_of(gv.cpu().numpy()).reshape(B, k)), f"largest={largest}"
