"""GPU parity: the CUDA library against the CPU oracle (bit-exact values and
index sets, lowest-position ties) and against the reference RadiK itself
(bit-exact value multisets, sorted sequences; RadiK's indices are a valid
selection).  All calls go through the C ABI (libradik_b200.so)."""
import numpy as np
import pytest

import oracle
from radik_b200 import workloads

from conftest import assert_same_selection, bits_of

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import radik_b200 as rk  # noqa: E402

DEV = "cuda:0"


def to_dev(x: np.ndarray, dtype: int):
    t = torch.from_numpy(np.ascontiguousarray(x))
    if dtype == rk.BF16:
        t = t.view(torch.bfloat16)
    return t.to(DEV)


def values_for(dtype, n, dist, seed):
    if dist == "normal":
        x = workloads.normal(n, seed)
    elif dist == "u01":
        x = workloads.uniform01(n, seed)
    elif dist == "ties":
        x = np.floor(workloads.normal(n, seed) * 3).astype(np.float32)
    elif dist == "zero":
        x = np.zeros(n, np.float32)
    elif dist in workloads.SKEW_DISTRIBUTIONS:
        x = workloads.skew_row(dist, n, seed)
    else:
        raise ValueError(dist)
    if dtype == rk.F16:
        return x.astype(np.float16)
    if dtype == rk.BF16:
        return workloads.to_bf16_bits(x)
    return x


def run_both(flat_np, lengths, k, dtype, largest, sorted_, ascend=None, scale=False, idx_in=None, idx64=False):
    t = to_dev(flat_np, dtype)
    tin = to_dev(idx_in, rk.F32) if idx_in is not None else None
    gv, gi = rk.topk(t, k, lengths, largest=largest, sorted=sorted_, ascend=ascend, with_scale=scale,
                     idx_in=tin, idx64=idx64)
    gv = gv.view(torch.int16) if dtype == rk.BF16 else gv
    gvn = gv.cpu().numpy().reshape(-1)
    gin = gi.cpu().numpy().reshape(-1)
    flags = oracle.flags_of(largest, sorted_, ascend, scale, idx_in is not None, idx64)
    ov, oi = oracle.topk(flat_np, lengths, k, flags=flags, dtype=dtype, idx_in=idx_in)
    if dtype == rk.BF16:
        gvn = gvn.view(np.uint16)
    return (gvn, gin), (ov, oi)


SHAPES = [
    # B, n, k
    (1, 1000, 10),          # smem row
    (5, 16384, 300),        # smem rows at the cap
    (3, 16385, 64),         # first multi-chunk rows
    (2, 100000, 256),
    (1, 1 << 20, 256),      # single-row benchmark shape
    (8, 1 << 20, 1024),
    (4, 300000, 4096),
    (2, 50000, 20000),      # one-CTA row, k > sort cap (merge sort path when sorted)
    (2, 1 << 20, 20000),    # radix grid rows (k * 64 > n)
    (3, 300000, 6000),      # radix grid rows just above the one-CTA cap
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"B{s[0]}-n{s[1]}-k{s[2]}")
@pytest.mark.parametrize("dtype", [rk.F32, rk.F16, rk.BF16], ids=["f32", "f16", "bf16"])
@pytest.mark.parametrize("largest,sorted_", [(True, False), (False, True), (True, True)])
def test_parity_vs_oracle(shape, dtype, largest, sorted_):
    B, n, k = shape
    flat = np.concatenate([values_for(dtype, n, "normal", 11 * r + n) for r in range(B)])
    got, want = run_both(flat, [n] * B, k, dtype, largest, sorted_)
    assert_same_selection(got, want, [n] * B, [k] * B, [r * k for r in range(B)], sorted_, f"{shape}")


@pytest.mark.parametrize("dist", ["u01", "ties", "zero", "mantissa_noise", "constant_heavy", "zipf"])
@pytest.mark.parametrize("n,k", [(70000, 100), (1 << 20, 2048), (20000, 5000), (1 << 20, 20000)])
def test_parity_distributions(dist, n, k):
    flat = values_for(rk.F32, n, dist, 5)
    for largest in (True, False):
        got, want = run_both(flat, [n], k, rk.F32, largest, True)
        assert_same_selection(got, want, [n], [k], [0], True, f"{dist} largest={largest}")


def test_parity_uneven_rows_and_idle_fill():
    lengths = [0, 1, 5, 16384, 16385, 100000, 3, 70001, 250000, 1 << 18]
    flat = np.concatenate([values_for(rk.F32, n, "normal", 3 + r) for r, n in enumerate(lengths)])
    k = 300
    for sorted_ in (False, True):
        got, want = run_both(flat, lengths, k, rk.F32, True, sorted_)
        assert_same_selection(got, want, lengths, [k] * len(lengths), [r * k for r in range(len(lengths))], sorted_)


@pytest.mark.parametrize("shape", [(300, 32768, 64), (512, 5000, 100), (200, 20000, 3000), (64, 8192, 8192)])
@pytest.mark.parametrize("dtype", [rk.F32, rk.F16])
def test_calls_of_short_rows_only(shape, dtype):
    # every row is selected by one team (smem or one-CTA rows): both the side
    # and the consumer teams take rows, the consumer team in the ring
    B, n, k = shape
    flat = np.concatenate([values_for(dtype, n, "normal", 80 + r) for r in range(B)])
    for largest, sorted_ in ((True, False), (False, True)):
        got, want = run_both(flat, [n] * B, k, dtype, largest, sorted_)
        assert_same_selection(got, want, [n] * B, [k] * B, [r * k for r in range(B)], sorted_)


def test_uneven_short_rows_only():
    lengths = [int(v) for v in workloads.rng(81).integers(1, 32768, size=300)]
    flat = np.concatenate([values_for(rk.F32, n, "ties", 90 + r) for r, n in enumerate(lengths)])
    k = 777
    for sorted_ in (False, True):
        got, want = run_both(flat, lengths, k, rk.F32, True, sorted_)
        assert_same_selection(got, want, lengths, [k] * len(lengths), [r * k for r in range(len(lengths))], sorted_)


@pytest.mark.parametrize("k", [2049, 4096, 5000, 8192])
def test_sorted_short_rows_with_large_k(k):
    # rows held in shared memory (n <= 8192) whose sorted outputs exceed
    # 2048 entries: the sort's scratch must stay inside the team's area
    lengths = [5000, 8192, 2500, 8000]
    flat = np.concatenate([values_for(rk.F32, n, "normal", 60 + r) for r, n in enumerate(lengths)])
    for largest in (True, False):
        got, want = run_both(flat, lengths, k, rk.F32, largest, True)
        assert_same_selection(got, want, lengths, [k] * len(lengths), [r * k for r in range(len(lengths))], True)


@pytest.mark.parametrize("dtype", [rk.F32, rk.F16])
def test_parity_withscale(dtype):
    g = workloads.rng(2)
    n = 200000
    x = (np.float32(0.6) + np.float32(0.1) * g.random(2 * n, dtype=np.float32))
    flat = x.astype(np.float16) if dtype == rk.F16 else x
    for largest, sorted_ in ((True, True), (False, False)):
        got, want = run_both(flat, [n, n], 700, dtype, largest, sorted_, scale=True)
        assert_same_selection(got, want, [n, n], [700, 700], [0, 700], sorted_)


@pytest.mark.parametrize("idx64", [False, True])
def test_parity_withidxin(idx64):
    n = [90000, 4000, 300000]
    flat = np.concatenate([values_for(rk.F32, m, "ties", 9 + r) for r, m in enumerate(n)])
    perm = workloads.rng(4).permutation(len(flat)).astype(np.int64 if idx64 else np.int32)
    got, want = run_both(flat, n, 777, rk.F32, True, True, idx_in=perm, idx64=idx64)
    assert_same_selection(got, want, n, [777] * 3, [0, 777, 1554], True)


def test_ascending_largest_and_descending_smallest():
    n = 123457
    flat = values_for(rk.F32, n, "ties", 1)
    for largest, ascend in ((True, True), (False, False)):
        got, want = run_both(flat, [n], 999, rk.F32, largest, True, ascend=ascend)
        assert_same_selection(got, want, [n], [999], [0], True)


def test_misaligned_row_starts():
    # odd row lengths put later rows at unaligned addresses
    lengths = [17, 100003, 65537, 99999, 3]
    for dtype in (rk.F32, rk.F16):
        flat = np.concatenate([values_for(dtype, m, "u01", 20 + r) for r, m in enumerate(lengths)])
        got, want = run_both(flat, lengths, 129, dtype, True, False)
        assert_same_selection(got, want, lengths, [129] * 5, [129 * r for r in range(5)], False)


def test_topk_rows_uneven_k():
    ns, ks = workloads.uneven_rows(64, 3, 10, 19, 2048)
    flat = np.concatenate([values_for(rk.F32, m, "normal", 40 + r) for r, m in enumerate(ns)])
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]])
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]])
    rows = [(int(a), int(b), int(n), int(k)) for a, b, n, k in zip(offs, oo, ns, ks)]
    for sorted_ in (False, True):
        gv, gi = rk.topk_rows(to_dev(flat, rk.F32), rows, largest=True, sorted=sorted_)
        flags = oracle.flags_of(True, sorted_)
        ov, oi = oracle.topk(flat, ns, ks, flags=flags, out_offsets=oo)
        assert_same_selection((gv.cpu().numpy(), gi.cpu().numpy()), (ov, oi), ns, ks, oo, sorted_)


def test_repeat_calls_are_identical():
    n = 1 << 20
    t = to_dev(values_for(rk.F32, 4 * n, "ties", 8), rk.F32)
    a = rk.topk(t, 512, [n] * 4, largest=True, sorted=True)
    b = rk.topk(t, 512, [n] * 4, largest=True, sorted=True)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_workspace_reuse_across_shapes():
    ws = torch.empty(rk.get_radix_select_l_workspace_size(rk.F32, 2048, 1 << 20, 16), dtype=torch.uint8, device=DEV)
    for (B, n, k) in ((16, 1 << 20, 2048), (3, 5000, 7), (16, 400000, 64)):
        flat = values_for(rk.F32, B * n, "normal", B + n)
        gv, gi = rk.topk(to_dev(flat, rk.F32), k, [n] * B, largest=True, sorted=True, workspace=ws)
        ov, oi = oracle.topk(flat, [n] * B, k, flags=oracle.flags_of(True, True))
        assert_same_selection((gv.cpu().numpy().reshape(-1), gi.cpu().numpy().reshape(-1)), (ov, oi), [n] * B,
                              [k] * B, [r * k for r in range(B)], True)


# ---------------------------------------------------------------------------
# against the reference RadiK on the same device buffers
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def ref():
    try:
        return oracle.RefRadik()
    except FileNotFoundError as e:
        pytest.skip(str(e))


@pytest.mark.parametrize("case", [
    (rk.F32, 1, 1 << 20, 256, True, False, False),
    (rk.F32, 16, 1 << 20, 1024, True, False, True),
    (rk.F32, 8, 1 << 20, 32, False, True, True),
    (rk.F16, 16, 1 << 20, 256, True, False, True),
    (rk.F32, 1, 1 << 22, 4096, True, False, True),
])
def test_value_multisets_match_reference_radik(ref, case):
    dtype, B, n, k, largest, ascend, sorted_ = case
    flat = np.concatenate([values_for(dtype, n, "u01", 1000 + r) for r in range(B)])
    t = to_dev(flat, dtype)
    vo = torch.zeros(B * k, dtype=t.dtype, device=DEV)
    io = torch.zeros(B * k, dtype=torch.int32, device=DEV)
    ws = torch.zeros(ref.workspace_size(dtype, k, n, B), dtype=torch.uint8, device=DEV)
    ref.topk(dtype, largest, ascend, False, sorted_, t.data_ptr(), vo.data_ptr(), io.data_ptr(), ws.data_ptr(),
             [n] * B, k, torch.cuda.current_stream().cuda_stream)
    gv, gi = rk.topk(t, k, [n] * B, largest=largest, sorted=sorted_, ascend=ascend)
    rv = bits_of(vo.cpu().numpy()).reshape(B, k)
    ri = io.cpu().numpy().reshape(B, k).astype(np.int64)
    ov = bits_of(gv.cpu().numpy()).reshape(B, k)
    rows = bits_of(flat).reshape(B, n)
    for r in range(B):
        assert np.array_equal(np.sort(rv[r]), np.sort(ov[r])), f"row {r} value multiset"
        if sorted_:
            assert np.array_equal(rv[r], ov[r]), f"row {r} sorted sequence"
        assert np.array_equal(rows[r][ri[r]], rv[r]) and len(np.unique(ri[r])) == k


@pytest.mark.parametrize("dist", ["mantissa_noise", "zipf", "constant_heavy", "zero"])
def test_phase_b_large_rows(dist):
    """Rows whose threshold misses or whose selected bin is huge finish in the
    multi-CTA levels; results must still be exact."""
    n = 1 << 22
    flat = values_for(rk.F32, n, dist, 77)
    for largest, k in ((False, 4096), (True, 100000), (True, 64)):
        got, want = run_both(flat, [n], k, rk.F32, largest, False)
        assert_same_selection(got, want, [n], [k], [0], False, f"{dist} largest={largest} k={k}")


def test_status_is_clean_after_calls():
    n = 1 << 20
    t = to_dev(values_for(rk.F32, 2 * n, "u01", 3), rk.F32)
    ws = torch.empty(rk.get_radix_select_l_workspace_size(rk.F32, 256, n, 2), dtype=torch.uint8, device=DEV)
    rk.topk(t, 256, [n, n], workspace=ws, check=False)
    assert rk.status(ws) == 0


def test_topk_rows_replayed_from_cuda_graph():
    """The one-launch uneven form takes device descriptors and never blocks the
    host, so it can be captured once and replayed on new data."""
    ns, ks = workloads.uneven_rows(48, 21, 10, 20, 2048)
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int64)
    total_n, total_out = int(sum(ns)), int(sum(ks))
    desc = np.zeros(len(ns), dtype=[("in_off", "<i8"), ("out_off", "<i8"), ("n", "<i4"), ("k", "<i4")])
    desc["in_off"], desc["out_off"], desc["n"], desc["k"] = offs, oo, ns, ks
    desc_dev = torch.from_numpy(desc.view(np.uint8).copy()).to(DEV)
    flags = rk.make_flags(True, True)
    ws = torch.empty(rk.get_rows_workspace_size(rk.F32, len(ns), total_n, max(ns), max(ks), flags),
                     dtype=torch.uint8, device=DEV)
    x = torch.empty(total_n, dtype=torch.float32, device=DEV)
    vals = torch.empty(total_out, dtype=torch.float32, device=DEV)
    idx = torch.empty(total_out, dtype=torch.int32, device=DEV)
    L = rk.lib()

    def call():
        rk._check(L.radik_topk_rows(rk.F32, flags, x.data_ptr(), None, vals.data_ptr(), idx.data_ptr(), ws.data_ptr(),
                                    ws.numel(), desc_dev.data_ptr(), len(ns), total_n, max(ns), max(ks),
                                    torch.cuda.current_stream().cuda_stream))

    x.copy_(torch.from_numpy(workloads.normal(total_n, 1)))
    call()  # first call on the device outside the capture (sets up the launch configuration)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        call()
    for seed in (2, 3):
        host = workloads.normal(total_n, seed)
        x.copy_(torch.from_numpy(host))
        graph.replay()
        torch.cuda.synchronize()
        assert rk.status(ws) == 0
        ov, oi = oracle.topk(host, ns, ks, flags=oracle.flags_of(True, True), out_offsets=[int(v) for v in oo])
        assert_same_selection((vals.cpu().numpy(), idx.cpu().numpy()), (ov, oi), ns, ks, oo, True, f"seed {seed}")


@pytest.mark.parametrize("shape", [(32, 1 << 20, 256), (2, 1 << 20, 20000), (16, 200000, 300)],
                         ids=["pref", "radix", "cta-cap"])
def test_autotune_keeps_results_exact(shape, tmp_path):
    """Whatever the tuner picks (chunk, first digit, CTA row cap), results
    stay bit-identical, and a saved table reloads to the same choice."""
    B, n, k = shape
    flat = np.concatenate([values_for(rk.F32, n, "normal", 900 + r) for r in range(B)])
    t = to_dev(flat, rk.F32).view(B, n)
    before = rk.topk(t, k, largest=True, sorted=True)
    try:
        c = rk.autotune(t, k, largest=True, sorted=True)
        assert c["ms"] > 0
        assert c["chunk"] == 0 or (4096 <= c["chunk"] <= (1 << 18) and c["chunk"] % 32 == 0)
        after = rk.topk(t, k, largest=True, sorted=True)
        assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])
        path = str(tmp_path / "tune.txt")
        rk.autotune_save(path)
        rk.autotune_reset()
        rk.autotune_load(path)
        again = rk.topk(t, k, largest=True, sorted=True)
        assert torch.equal(before[0], again[0]) and torch.equal(before[1], again[1])
    finally:
        rk.autotune_reset()


def test_autotune_rows_keeps_results_exact():
    ns, ks = workloads.uneven_rows(96, 5, 10, 20, 2048)
    flat = np.concatenate([values_for(rk.F32, m, "normal", 70 + r) for r, m in enumerate(ns)])
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]])
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]])
    rows = [(int(a), int(b), int(n), int(k)) for a, b, n, k in zip(offs, oo, ns, ks)]
    x = to_dev(flat, rk.F32)
    host = (rk.RowDesc * len(rows))(*[rk.RowDesc(*r) for r in rows])
    desc = torch.frombuffer(bytearray(bytes(host)), dtype=torch.uint8).to(DEV)
    bounds = (sum(ns), max(ns), max(ks))
    try:
        c = rk.autotune_rows(x, desc, len(rows), bounds, int(sum(ks)), largest=True)
        assert c["ms"] > 0
        gv, gi = rk.topk_rows(x, rows, largest=True)
        ov, oi = oracle.topk(flat, ns, ks, flags=oracle.flags_of(True, False), out_offsets=oo)
        assert_same_selection((gv.cpu().numpy(), gi.cpu().numpy()), (ov, oi), ns, ks, oo, False)
    finally:
        rk.autotune_reset()


@pytest.mark.parametrize("dist", ["u01", "zipf", "mantissa_noise"])
@pytest.mark.parametrize("k", [256, 4096])
def test_single_huge_row(dist, k):
    """One 2^24-key row: the kernel's first sample is a large one taken by the
    whole CTA, and the row's finish runs on an idle consumer team."""
    n = 1 << 24
    flat = values_for(rk.F32, n, dist, 123)
    for largest in (True, False):
        got, want = run_both(flat, [n], k, rk.F32, largest, True)
        assert_same_selection(got, want, [n], [k], [0], True, f"{dist} largest={largest}")


def test_uneven_lengths_refuse_stream_capture():
    """radik_topk copies the descriptors of unequal rows from host memory that
    lives only for the call, so a capture of it is refused (RADIK_ENOTSUP);
    radik_topk_rows, with device descriptors, is the capturable form."""
    lengths = [5000, 70000, 300]
    x = to_dev(values_for(rk.F32, sum(lengths), "normal", 1), rk.F32)
    rk.topk(x, 10, lengths)  # outside a capture: fine
    graph = torch.cuda.CUDAGraph()
    with pytest.raises(rk.RadikError) as err:
        with torch.cuda.graph(graph):
            rk.topk(x, 10, lengths, check=False)
    assert err.value.code == rk.ENOTSUP


@pytest.mark.parametrize("dist", ["zero", "mantissa_noise", "constant_heavy", "ties"])
def test_several_rows_in_phase_b(dist):
    """Several rows of one batch whose sampled threshold catches too many keys
    (ties) finish together in the grid-wide phase B."""
    n, B = 1 << 21, 3
    flat = np.concatenate([values_for(rk.F32, n, dist, 50 + r) for r in range(B)])
    for largest, k in ((True, 100), (False, 3000), (True, 20000)):
        got, want = run_both(flat, [n] * B, k, rk.F32, largest, True)
        assert_same_selection(got, want, [n] * B, [k] * B, [r * k for r in range(B)], True, f"{dist} k={k}")
