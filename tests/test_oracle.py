"""CPU tests of the oracle (the CPU restatement of RadiK's selection).

* An independent numpy restatement of the same rule (order-preserving key,
  largest/smallest flip, WITHSCALE difference, lowest-position ties) must
  agree with the C++ oracle bit for bit.
* Golden vectors produced by the reference RadiK itself on a B200
  (tests/golden/make_golden.py) pin the oracle: value multisets bit-exact,
  sorted value sequences bit-exact, and every RadiK index must point at its
  value.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from radik_b200 import workloads

from conftest import assert_same_selection, bits_of

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def np_keys(vals: np.ndarray, dtype: int, flags: int) -> np.ndarray:
    """numpy restatement of the selection key (smaller = better)."""
    if flags & oracle.WITHSCALE:
        if dtype == oracle.BF16:
            f = (vals.astype(np.uint32) << 16).view(np.float32)
        else:
            f = vals.astype(np.float32)
        s = f[0] if len(f) else np.float32(0)
        if not np.isfinite(s):
            s = np.float32(0)
        u = (f - np.float32(s)).astype(np.float32).view(np.uint32)
        k = np.where(u >> 31, ~u, u | np.uint32(0x80000000)).astype(np.uint32)
        return (~k).astype(np.uint64) & 0xFFFFFFFF if flags & oracle.LARGEST else k.astype(np.uint64)
    if dtype == oracle.F32:
        u = vals.view(np.uint32)
        k = np.where(u >> 31, ~u, u | np.uint32(0x80000000)).astype(np.uint32)
        return (~k).astype(np.uint64) & 0xFFFFFFFF if flags & oracle.LARGEST else k.astype(np.uint64)
    u = vals.view(np.uint16).astype(np.uint32)
    k = np.where(u >> 15, (~u) & 0xFFFF, u | 0x8000).astype(np.uint32)
    return ((~k) & 0xFFFF).astype(np.uint64) if flags & oracle.LARGEST else k.astype(np.uint64)


def np_topk_row(vals: np.ndarray, k: int, dtype: int, flags: int):
    n = len(vals)
    kk = min(n, k)
    keys = np_keys(vals, dtype, flags)
    comp = (keys << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    sel = np.sort(comp)[:kk]
    pos = (sel & np.uint64(0xFFFFFFFF)).astype(np.int64)
    if flags & oracle.SORTED:
        b = vals.view(np.uint32) if dtype == oracle.F32 else vals.view(np.uint16).astype(np.uint32)
        b = b[pos]
        if dtype == oracle.F32:
            ok = np.where(b >> 31, ~b, b | np.uint32(0x80000000)).astype(np.uint64)
            if not flags & oracle.ASCEND:
                ok = (~ok) & np.uint64(0xFFFFFFFF)
        else:
            ok = np.where(b >> 15, (~b) & 0xFFFF, b | 0x8000).astype(np.uint64)
            if not flags & oracle.ASCEND:
                ok = (~ok) & np.uint64(0xFFFF)
        pos = pos[np.lexsort((pos, ok))]
    else:
        pos = np.sort(pos)
    return pos


CASES = [
    # dtype, B, n, k, distribution
    (oracle.F32, 3, 1000, 10, "normal"),
    (oracle.F32, 2, 5000, 300, "ties"),
    (oracle.F32, 1, 300000, 256, "uniform"),
    (oracle.F16, 4, 3000, 64, "normal"),
    (oracle.F16, 2, 20000, 500, "uniform"),
    (oracle.BF16, 3, 4000, 33, "normal"),
    (oracle.F32, 2, 50, 80, "normal"),   # n < k: idle fill
]


def make_values(dtype, n, dist, seed):
    if dist == "normal":
        x = workloads.normal(n, seed)
    elif dist == "ties":
        x = np.floor(workloads.normal(n, seed) * 4).astype(np.float32)
    else:
        x = workloads.uniform01(n, seed)
    if dtype == oracle.F16:
        return x.astype(np.float16)
    if dtype == oracle.BF16:
        return workloads.to_bf16_bits(x)
    return x


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"dt{c[0]}-B{c[1]}-n{c[2]}-k{c[3]}-{c[4]}")
@pytest.mark.parametrize("largest,sorted_,ascend,scale", [
    (True, False, False, False), (False, False, True, False), (True, True, False, False),
    (False, True, True, False), (True, True, True, False), (True, False, False, True), (False, True, True, True)])
def test_oracle_matches_numpy_restatement(case, largest, sorted_, ascend, scale):
    dtype, B, n, k, dist = case
    flags = oracle.flags_of(largest, sorted_, ascend, scale)
    rows = [make_values(dtype, n, dist, 100 + r) for r in range(B)]
    flat = np.concatenate(rows)
    vout, iout = oracle.topk(flat, [n] * B, k, flags=flags, dtype=dtype)
    for r in range(B):
        pos = np_topk_row(rows[r], k, dtype, flags)
        kk = len(pos)
        assert np.array_equal(iout[r * k:r * k + kk], pos), f"row {r}"
        want_bits = bits_of(rows[r])[pos]
        assert np.array_equal(bits_of(vout)[r * k:r * k + kk], want_bits)
        assert np.all(iout[r * k + kk:(r + 1) * k] == -1)


def test_oracle_uneven_rows_and_idx_in():
    g = workloads.rng(7)
    lengths = [0, 1, 17, 4096, 30001, 5]
    ks = [3, 1, 17, 100, 2048, 9]
    flat = workloads.normal(sum(lengths), 3)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]])
    idx_in = g.permutation(len(flat)).astype(np.int64)
    flags = oracle.flags_of(True, True, False, False, True, True)
    v, i = oracle.topk(flat, lengths, ks, flags=flags, idx_in=idx_in, out_offsets=oo)
    off = 0
    for r, (n, k) in enumerate(zip(lengths, ks)):
        row = flat[off:off + n]
        pos = np_topk_row(row, k, oracle.F32, flags)
        kk = len(pos)
        assert np.array_equal(i[oo[r]:oo[r] + kk], idx_in[off + pos])
        assert np.all(i[oo[r] + kk:oo[r] + k] == -1)
        off += n


def test_oracle_thread_count_does_not_change_result():
    x = workloads.uniform01(1 << 20, 0)
    f = oracle.flags_of(True, False)
    a = oracle.topk(x, [len(x)], 256, flags=f, nthreads=1)
    b = oracle.topk(x, [len(x)], 256, flags=f, nthreads=8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_select_key_order():
    # -0.0 < +0.0 and NaN above +inf for the unflipped key
    f = oracle.flags_of(False)
    k = lambda x: oracle.select_key(oracle.F32, f, int(np.float32(x).view(np.uint32)))
    assert k(-1.0) < k(-0.0) < k(0.0) < k(1e-30) < k(np.inf) < k(np.nan)


def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def test_golden_fixtures_present():
    assert _golden_files(), "tests/golden holds the RadiK-produced fixtures"


@pytest.mark.parametrize("path", _golden_files(), ids=os.path.basename)
def test_oracle_matches_radik_golden(path):
    """The oracle reproduces what the reference RadiK returned on a B200."""
    z = np.load(path)
    dtype = int(z["dtype"])
    flags = int(z["flags"])
    lengths = [int(x) for x in z["lengths"]]
    K = int(z["K"])
    vals = z["values"]
    vout, iout = oracle.topk(vals, lengths, K, flags=flags, dtype=dtype)
    rv = z["ref_vals"]
    ri = z["ref_idx"]
    off = 0
    for r, n in enumerate(lengths):
        kk = min(n, K)
        ob = bits_of(vout)[r * K:r * K + kk]
        rb = bits_of(rv)[r * K:r * K + kk]
        # value multisets are bit-exact
        assert np.array_equal(np.sort(ob), np.sort(rb)), f"{path} row {r}: value multiset"
        if flags & oracle.SORTED:
            # sorted sequences are bit-exact position by position
            assert np.array_equal(ob, rb), f"{path} row {r}: sorted sequence"
        # RadiK's indices point at their values (ties may pick other positions)
        row_bits = bits_of(vals)[off:off + n]
        ridx = ri[r * K:r * K + kk].astype(np.int64)
        assert np.all((ridx >= 0) & (ridx < n))
        assert np.array_equal(row_bits[ridx], rb)
        assert len(np.unique(ridx)) == kk
        off += n
