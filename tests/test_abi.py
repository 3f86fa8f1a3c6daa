"""CPU tests of the C ABI: the library loads, exports every declared entry
point, and rejects bad arguments before touching the device (no GPU needed)."""
import ctypes
import os
import re

import pytest

import radik_b200 as rk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("radik_b200.h",):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(radik_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_declared_symbols():
    lib = rk.lib()
    names = declared_functions()
    assert "radik_topk" in names and "radik_get_workspace_size" in names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"


def test_version_and_strerror():
    assert rk.lib().radik_version() >= 100
    for code in range(7):
        assert rk.lib().radik_strerror(code)


def test_workspace_size_is_below_reference_formula():
    # RadiK: B * (4 * 4096 + 2 * 4 * n + 20) + 4 * (B + 1)  (topk_radixselect.h:22-33)
    B, n, K = 256, 1 << 20, 256
    ours = rk.get_radix_select_l_workspace_size(rk.F32, K, n, B, rk.SORTED)
    ref = B * (4 * 4096 + 8 * n + 20) + 4 * (B + 1)
    assert 0 < ours < ref


def test_workspace_size_monotone():
    a = rk.get_radix_select_l_workspace_size(rk.F32, 256, 1 << 16, 8)
    b = rk.get_radix_select_l_workspace_size(rk.F32, 256, 1 << 20, 8)
    c = rk.get_radix_select_l_workspace_size(rk.F32, 256, 1 << 20, 16)
    assert a <= b <= c
    s = rk.get_radix_select_l_workspace_size(rk.F32, 1 << 16, 1 << 24, 1, rk.SORTED)
    u = rk.get_radix_select_l_workspace_size(rk.F32, 1 << 16, 1 << 24, 1, 0)
    assert s > u  # merge-sort scratch for k > 4096


def _call(dtype=rk.F32, flags=0, ws=1 << 12, val=1 << 12, out=1 << 12, idx_in=None, lens=(10,), K=4):
    arr = (ctypes.c_int * len(lens))(*lens)
    return rk.lib().radik_topk(dtype, flags, val, idx_in, out, out, ws, 1 << 30, arr, len(lens), K, None)


def test_rejects_bad_arguments_without_device():
    assert _call(ws=None) == rk.EWORKSPACE
    assert _call(ws=(1 << 12) + 8) == rk.EWORKSPACE  # unaligned workspace
    assert _call(dtype=7) == rk.EINVAL
    assert _call(flags=1 << 10) == rk.EINVAL
    assert _call(K=-1) == rk.EINVAL
    assert _call(lens=(-3,)) == rk.EINVAL
    assert _call(flags=rk.WITHIDXIN) == rk.EINVAL
    assert _call(val=None) == rk.EINVAL
    assert "null" in rk.lib().radik_last_error().decode()
    assert _call(ws=None) == rk.EWORKSPACE
    assert "workspace" in rk.lib().radik_last_error().decode()


def test_empty_batch_is_a_no_op():
    assert _call(lens=(), K=4) == rk.OK
    assert _call(K=0) == rk.OK


def test_get_status_needs_workspace():
    assert rk.lib().radik_get_status(None, None, None) == rk.EWORKSPACE


def test_flag_helper():
    f = rk.make_flags(largest=True, sorted=True)
    assert f == rk.LARGEST | rk.SORTED
    assert rk.make_flags(largest=False) == rk.ASCEND


def test_autotune_rejects_empty_call_without_device():
    arr = (ctypes.c_int * 1)(0)
    rc = rk.lib().radik_autotune(rk.F32, 0, 1 << 12, None, 1 << 12, 1 << 12, 1 << 12, 1 << 20, arr, 0, 4, None, None)
    assert rc == rk.EINVAL


def test_tuning_table_round_trip_without_device(tmp_path):
    """radik_autotune_load / _save: a table of buckets reloads unchanged; a
    malformed one is rejected."""
    good = tmp_path / "t.txt"
    good.write_text("# comment\n14208 0 0 65536\n24280 65536 11 131072\n")
    try:
        rk.autotune_load(str(good))
        out = tmp_path / "u.txt"
        rk.autotune_save(str(out))
        lines = [l for l in out.read_text().splitlines() if not l.startswith("#")]
        assert lines == ["14208 0 0 65536", "24280 65536 11 131072"]
        bad = tmp_path / "b.txt"
        bad.write_text("14208 0 0\n")
        with pytest.raises(rk.RadikError):
            rk.autotune_load(str(bad))
        bad.write_text("14208 1000 0 0\n")  # chunk below the 4096-key minimum
        with pytest.raises(rk.RadikError):
            rk.autotune_load(str(bad))
    finally:
        rk.autotune_reset()
