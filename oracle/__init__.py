"""Test-only checkers for radik_b200.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py
(its CPU-baseline leg and its reference arm) may import this package; the
library never does.

* ``topk``      -- the CPU restatement of RadiK's selection (liboracle.so built
                   from topk_oracle.cpp; exact, lowest-position ties).  Parity
                   is pinned by tests/test_oracle.py against golden vectors
                   that the reference RadiK itself produced
                   (tests/golden/make_golden.py).
* ``RefRadik``  -- the unmodified reference RadiK compiled from its sources
                   (oracle/_ref/libradik_ref.so), callable on torch CUDA
                   tensors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libradik_ref.so")

F32, F16, BF16 = 0, 1, 2
LARGEST, SORTED, ASCEND, WITHSCALE, WITHIDXIN, IDX64 = 1, 2, 4, 8, 16, 32

_oracle = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def _load_oracle() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        vp = ctypes.c_void_p
        L.oracle_topk.argtypes = [ctypes.c_int, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int]
        L.oracle_topk.restype = ctypes.c_int
        L.oracle_select_key.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float]
        L.oracle_select_key.restype = ctypes.c_uint32
        L.oracle_key_bits.argtypes = [ctypes.c_int, ctypes.c_uint32]
        L.oracle_key_bits.restype = ctypes.c_int
        L.oracle_max_threads.restype = ctypes.c_int
        _oracle = L
    return _oracle


def max_threads() -> int:
    return _load_oracle().oracle_max_threads()


def flags_of(largest=True, sorted=False, ascend=None, with_scale=False, with_idx_in=False, idx64=False) -> int:
    if ascend is None:
        ascend = not largest
    return ((LARGEST if largest else 0) | (SORTED if sorted else 0) | (ASCEND if ascend else 0)
            | (WITHSCALE if with_scale else 0) | (WITHIDXIN if with_idx_in else 0) | (IDX64 if idx64 else 0))


def _dtype_code(arr: np.ndarray, dtype: Optional[int]) -> int:
    if dtype is not None:
        return dtype
    if arr.dtype == np.float32:
        return F32
    if arr.dtype == np.float16:
        return F16
    raise ValueError("pass dtype=BF16 for bfloat16 bit patterns held as uint16")


def topk(values: np.ndarray, lengths: Sequence[int], k, *, flags: int, dtype: Optional[int] = None,
         idx_in: Optional[np.ndarray] = None, out_offsets: Optional[Sequence[int]] = None,
         out_size: Optional[int] = None, nthreads: int = 0):
    """Exact batched top-k on the CPU.

    values: 1-D, rows back to back (float32, float16, or uint16 bf16 bits with
    dtype=BF16).  k: int or per-row sequence.  Output row r starts at
    out_offsets[r] (default r * k for a uniform k).  Returns flat
    (vals, idx) arrays; unsorted rows are in ascending position order.
    """
    L = _load_oracle()
    dt = _dtype_code(values, dtype)
    vals = np.ascontiguousarray(values)
    B = len(lengths)
    row_off = np.zeros(B + 1, dtype=np.int64)
    row_off[1:] = np.cumsum(np.asarray(lengths, dtype=np.int64))
    if np.isscalar(k):
        ks = np.full(B, int(k), dtype=np.int32)
    else:
        ks = np.asarray(k, dtype=np.int32)
    if out_offsets is None:
        oo = np.zeros(B, dtype=np.int64)
        if B > 1:
            oo[1:] = np.cumsum(ks[:-1].astype(np.int64)) if not np.isscalar(k) else np.arange(1, B) * int(k)
    else:
        oo = np.asarray(out_offsets, dtype=np.int64)
    total = int(out_size) if out_size is not None else int((oo + ks).max()) if B else 0
    es_dtype = vals.dtype if dt == F32 else np.uint16 if dt == BF16 else np.float16
    vout = np.zeros(max(total, 1), dtype=es_dtype)
    iout = np.zeros(max(total, 1), dtype=np.int64 if flags & IDX64 else np.int32)
    ii = None
    if flags & WITHIDXIN:
        ii = np.ascontiguousarray(idx_in, dtype=np.int64 if flags & IDX64 else np.int32)
    rc = L.oracle_topk(dt, flags, vals.ctypes.data, ii.ctypes.data if ii is not None else None,
                       row_off.ctypes.data, ks.ctypes.data, oo.ctypes.data, B,
                       vout.ctypes.data, iout.ctypes.data, nthreads)
    if rc != 0:
        raise ValueError("oracle_topk: bad arguments")
    return vout[:total], iout[:total]


def select_key(dtype: int, flags: int, bits: int, scaler: float = 0.0) -> int:
    return _load_oracle().oracle_select_key(dtype, flags, bits, scaler)


class RefRadik:
    """The reference RadiK (topKRadixSelectL) built from its own sources."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle ref, with the reference sources present)")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.ref_radik_workspace_size.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_size_t)]
        L.ref_radik_topk.argtypes = [ctypes.c_int] * 6 + [vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]
        L.ref_radik_last_error.restype = ctypes.c_char_p
        self.L = L

    def workspace_size(self, dtype: int, K: int, n_max: int, task_num: int) -> int:
        out = ctypes.c_size_t(0)
        if self.L.ref_radik_workspace_size(dtype, K, n_max, task_num, ctypes.byref(out)) != 0:
            raise ValueError("ref workspace size failed")
        return out.value

    def topk(self, dtype: int, largest: bool, ascend: bool, with_scale: bool, sorted: bool, val_in_ptr: int,
             val_out_ptr: int, idx_out_ptr: int, ws_ptr: int, task_len: Sequence[int], K: int, stream: int,
             idx_in_ptr: Optional[int] = None) -> None:
        n = len(task_len)
        arr = (ctypes.c_int * max(n, 1))(*[int(x) for x in task_len])
        rc = self.L.ref_radik_topk(dtype, int(largest), int(ascend), int(with_scale), int(idx_in_ptr is not None),
                                   int(sorted), val_in_ptr, idx_in_ptr, val_out_ptr, idx_out_ptr, ws_ptr, arr, n,
                                   int(K), stream)
        if rc != 0:
            raise RuntimeError(self.L.ref_radik_last_error().decode())
