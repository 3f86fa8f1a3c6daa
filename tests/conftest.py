import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def bits_of(a: np.ndarray) -> np.ndarray:
    """Raw bit patterns of a value array (uint32 for 4-byte, uint16 for 2-byte)."""
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype.itemsize == 4 else a.view(np.uint16)


def canonical_rows(vals: np.ndarray, idx: np.ndarray, lengths, ks, out_offsets, sorted_out: bool):
    """Per row: (value bits, indices) of the min(n, k) results, ordered by index
    when the output is unsorted, plus the idle-fill slots."""
    vb = bits_of(vals)
    rows = []
    for n, k, o in zip(lengths, ks, out_offsets):
        kk = min(n, k)
        v = vb[o:o + kk]
        i = idx[o:o + kk].astype(np.int64)
        if not sorted_out:
            order = np.argsort(i, kind="stable")
            v, i = v[order], i[order]
        rows.append((v, i, vb[o + kk:o + k], idx[o + kk:o + k].astype(np.int64)))
    return rows


def assert_same_selection(got, want, lengths, ks, out_offsets, sorted_out: bool, label: str = ""):
    g = canonical_rows(*got, lengths, ks, out_offsets, sorted_out)
    w = canonical_rows(*want, lengths, ks, out_offsets, sorted_out)
    for r, (a, b) in enumerate(zip(g, w)):
        assert np.array_equal(a[1], b[1]), f"{label} row {r}: indices differ (first diff at {np.argmax(a[1] != b[1]) if a[1].shape == b[1].shape else 'shape'})"
        assert np.array_equal(a[0], b[0]), f"{label} row {r}: value bits differ"
        assert np.all(a[3] == -1), f"{label} row {r}: idle slots must hold index -1"
        assert np.all(a[2] == 0), f"{label} row {r}: idle slots must hold value 0"
