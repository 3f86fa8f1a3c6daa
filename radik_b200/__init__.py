"""radik_b200 -- B200-native radix top-k selection.

Python host mirror of RadiK's entry points (leefige/radik,
radik/RadixSelect/topk_radixselect.h) over the library's C ABI
(include/radik_b200.h).  PyTorch supplies device memory and streams; the
selection itself runs in the in-tree CUDA library ``libradik_b200.so``.  There
is no fallback: if the library is missing, importing the bindings raises.

Reference mapping:
  getRadixSelectLWorkSpaceSize<ValType>(K, n, taskNum, &bytes)
      -> get_radix_select_l_workspace_size(dtype, K, n, task_num, ...)
  topKRadixSelectL<IdxType, LARGEST, ASCEND, WITHSCALE, WITHIDXIN>(
      valIn, idxIn, valOut, idxOut, workSpace, taskLen, taskNum, K, stream,
      needSorting)
      -> topk_radix_select_l(val_in, idx_in, val_out, idx_out, workspace,
                             task_len, K, largest=, ascend=, with_scale=,
                             with_idx_in=, need_sorting=, stream=)
  std::runtime_error -> RadikError
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libradik_b200.so")

F32, F16, BF16 = 0, 1, 2
LARGEST, SORTED, ASCEND, WITHSCALE, WITHIDXIN, IDX64 = 1, 2, 4, 8, 16, 32

OK, EINVAL, EWORKSPACE, ECUDA, ETIMEOUT, EINTERNAL, ENOTSUP = range(7)


class RadikError(RuntimeError):
    """A non-zero status from the library (RadiK raises std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"radik_b200 error {code}: {msg}")
        self.code = code


class RowDesc(ctypes.Structure):
    _fields_ = [("in_off", ctypes.c_int64), ("out_off", ctypes.c_int64), ("n", ctypes.c_int32), ("k", ctypes.c_int32)]


class TuneChoice(ctypes.Structure):
    """radik_tune_choice: a tuned bucket's knobs (0: built-in)."""
    _fields_ = [("chunk", ctypes.c_int), ("d1", ctypes.c_int), ("cta_cap", ctypes.c_int), ("ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"radik_b200: {LIB_PATH} is missing; build it with `python -m radik_b200.build` "
            "(there is no CPU fallback)"
        )
    L = ctypes.CDLL(LIB_PATH)
    vp, u32, i32, i64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int64, ctypes.c_size_t
    L.radik_get_workspace_size.argtypes = [i32, u32, i32, i32, i32, ctypes.POINTER(sz)]
    L.radik_get_workspace_size_rows.argtypes = [i32, u32, i32, i64, i32, i32, ctypes.POINTER(sz)]
    L.radik_topk.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_int), i32, i32, vp]
    L.radik_topk_rows.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, vp, i32, i64, i32, i32, vp]
    L.radik_topk_rows_ctas.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, vp, i32, i64, i32, i32, i32, vp]
    L.radik_engine_ctas.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.radik_get_call_span.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.radik_get_status.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int)]
    L.radik_autotune.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_int), i32, i32, vp,
                                 ctypes.POINTER(ctypes.c_int)]
    L.radik_autotune.restype = ctypes.c_int
    L.radik_autotune_reset.argtypes = []
    L.radik_autotune_reset.restype = None
    L.radik_autotune_ex.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_int), i32, i32, vp,
                                    ctypes.POINTER(TuneChoice)]
    L.radik_autotune_rows.argtypes = [i32, u32, vp, vp, vp, vp, vp, sz, vp, i32, i64, i32, i32, vp,
                                      ctypes.POINTER(TuneChoice)]
    L.radik_autotune_save.argtypes = [ctypes.c_char_p]
    L.radik_autotune_load.argtypes = [ctypes.c_char_p]
    L.radik_topk_static.argtypes = [i32, u32, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int), i32, i32, vp,
                                    ctypes.POINTER(vp)]
    L.radik_strerror.argtypes = [i32]
    L.radik_strerror.restype = ctypes.c_char_p
    L.radik_last_error.argtypes = []
    L.radik_last_error.restype = ctypes.c_char_p
    L.radik_timeline_attach.argtypes = [vp]
    L.radik_timeline_attach.restype = ctypes.c_int
    L.radik_version.argtypes = []
    for name in ("radik_get_workspace_size", "radik_get_workspace_size_rows", "radik_topk", "radik_topk_rows",
                 "radik_topk_rows_ctas", "radik_engine_ctas", "radik_get_call_span",
                 "radik_get_status", "radik_version", "radik_topk_static", "radik_autotune_ex", "radik_autotune_rows",
                 "radik_autotune_save", "radik_autotune_load"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _check(code: int) -> None:
    if code != OK:
        msg = lib().radik_last_error().decode(errors="replace")
        raise RadikError(code, msg or lib().radik_strerror(code).decode())


def dtype_code(torch_dtype) -> int:
    import torch

    m = {torch.float32: F32, torch.float16: F16, torch.bfloat16: BF16}
    if torch_dtype not in m:
        raise RadikError(EINVAL, f"unsupported value dtype {torch_dtype}")
    return m[torch_dtype]


def make_flags(largest: bool = True, sorted: bool = False, ascend: Optional[bool] = None,
               with_scale: bool = False, with_idx_in: bool = False, idx64: bool = False) -> int:
    """Flag bits; ascend defaults to the natural order (descending for largest)."""
    if ascend is None:
        ascend = not largest
    f = 0
    f |= LARGEST if largest else 0
    f |= SORTED if sorted else 0
    f |= ASCEND if ascend else 0
    f |= WITHSCALE if with_scale else 0
    f |= WITHIDXIN if with_idx_in else 0
    f |= IDX64 if idx64 else 0
    return f


def get_radix_select_l_workspace_size(dtype: int, K: int, n: int, task_num: int, flags: int = SORTED) -> int:
    """Bytes of workspace for topk_radix_select_l (getRadixSelectLWorkSpaceSize)."""
    out = ctypes.c_size_t(0)
    _check(lib().radik_get_workspace_size(dtype, flags, K, n, task_num, ctypes.byref(out)))
    return out.value


def get_rows_workspace_size(dtype: int, task_num: int, total_n: int, n_max: int, k_max: int, flags: int = SORTED) -> int:
    out = ctypes.c_size_t(0)
    _check(lib().radik_get_workspace_size_rows(dtype, flags, task_num, total_n, n_max, k_max, ctypes.byref(out)))
    return out.value


def _stream_handle(stream, device=None) -> Optional[int]:
    """The raw handle of ``stream``; None means the current stream of
    ``device`` (the current device when that is None too)."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(device)
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _device_of(t):
    """A context that makes ``t``'s CUDA device current for the C calls: the
    library launches on, and looks its static scratch up on, the current
    device, so a tensor on cuda:1 must not run while cuda:0 is current."""
    import torch

    if not t.is_cuda:
        raise RadikError(EINVAL, f"values must be a CUDA tensor (got device {t.device})")
    return torch.cuda.device(t.device)


def _same_device(values, *others) -> None:
    for o in others:
        if o is not None and o.device != values.device:
            raise RadikError(EINVAL, f"tensors on {o.device} and {values.device}: all must be on one device")


def topk_radix_select_l(val_in, idx_in, val_out, idx_out, workspace, task_len: Sequence[int], K: int, *,
                        largest: bool, ascend: bool, with_scale: bool = False, with_idx_in: bool = False,
                        need_sorting: bool = True, stream=None, idx64: Optional[bool] = None) -> None:
    """Mirror of topKRadixSelectL (topk_radixselect.h:59-70) on torch CUDA tensors.

    val_in holds the rows back to back; val_out/idx_out are task_num x K;
    task_len is a host sequence of row lengths.  Asynchronous on ``stream``.
    """
    import torch

    if workspace is None:
        raise RadikError(EWORKSPACE, "radix topk: workspace should not be null")
    if idx64 is None:
        idx64 = idx_out.dtype == torch.int64
    flags = make_flags(largest, need_sorting, ascend, with_scale, with_idx_in, idx64)
    n = len(task_len)
    arr = (ctypes.c_int * max(n, 1))(*[int(x) for x in task_len])
    _same_device(val_in, idx_in, val_out, idx_out, workspace)
    with _device_of(val_in):
        _check(lib().radik_topk(
            dtype_code(val_in.dtype), flags, val_in.data_ptr(), idx_in.data_ptr() if idx_in is not None else None,
            val_out.data_ptr(), idx_out.data_ptr(), workspace.data_ptr(),
            workspace.numel() * workspace.element_size(), arr, n, int(K), _stream_handle(stream, val_in.device)))


def status(workspace, stream=None) -> int:
    """Synchronise ``stream`` and raise RadikError if the last call failed on the device."""
    bits = ctypes.c_int(0)
    with _device_of(workspace):
        _check(lib().radik_get_status(workspace.data_ptr(), _stream_handle(stream, workspace.device),
                                      ctypes.byref(bits)))
    return bits.value


def call_span(workspace, stream=None) -> Tuple[int, int]:
    """(start_ns, end_ns): the GPU global-timer span of the selection kernel
    of the last call made with ``workspace`` (radik_get_call_span).
    Synchronises ``stream``."""
    t0, t1 = ctypes.c_uint64(0), ctypes.c_uint64(0)
    with _device_of(workspace):
        _check(lib().radik_get_call_span(workspace.data_ptr(), _stream_handle(stream, workspace.device),
                                         ctypes.byref(t0), ctypes.byref(t1)))
    return t0.value, t1.value


def topk(values, k: int, lengths: Optional[Sequence[int]] = None, *, largest: bool = True, sorted: bool = False,
         ascend: Optional[bool] = None, with_scale: bool = False, idx_in=None, idx64: bool = False,
         workspace=None, stream=None, check: bool = True) -> Tuple["object", "object"]:
    """Batched top-k of torch CUDA values.

    values: 2-D (rows of equal length) or 1-D with ``lengths`` (rows back to
    back).  Returns (vals[B, k], idx[B, k]); indices are positions in each row
    (or idx_in entries).  ``check`` synchronises and raises on a device error.
    """
    import torch

    if values.dim() == 2:
        B, n = values.shape
        lengths = [n] * B
        flat = values.contiguous().view(-1)
    else:
        if lengths is None:
            lengths = [values.numel()]
        flat = values.contiguous()
        B = len(lengths)
    flags = make_flags(largest, sorted, ascend, with_scale, idx_in is not None, idx64)
    dt = dtype_code(values.dtype)
    n_max = max(lengths) if lengths else 0
    _same_device(values, idx_in, workspace)
    with _device_of(values):
        if workspace is None:
            ws_bytes = get_radix_select_l_workspace_size(dt, k, n_max, B, flags)
            workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=values.device)
        vals = torch.empty((B, k), dtype=values.dtype, device=values.device)
        idx = torch.empty((B, k), dtype=torch.int64 if idx64 else torch.int32, device=values.device)
        arr = (ctypes.c_int * max(B, 1))(*[int(x) for x in lengths])
        _check(lib().radik_topk(dt, flags, flat.data_ptr(), idx_in.data_ptr() if idx_in is not None else None,
                                vals.data_ptr(), idx.data_ptr(), workspace.data_ptr(), workspace.numel(),
                                arr, B, int(k), _stream_handle(stream, values.device)))
    if check:
        status(workspace, stream)
    return vals, idx


def engine_ctas(device=None) -> int:
    """Engine CTAs (one per SM) a call on ``device`` can use at most."""
    import torch

    out = ctypes.c_int(0)
    with torch.cuda.device(device if device is not None else torch.cuda.current_device()):
        _check(lib().radik_engine_ctas(ctypes.byref(out)))
    return out.value


def topk_rows(values, rows, *, largest: bool = True, sorted: bool = False, ascend: Optional[bool] = None,
              with_scale: bool = False, idx_in=None, idx64: bool = False, total_out: Optional[int] = None,
              bounds: Optional[Tuple[int, int, int]] = None, workspace=None, stream=None, check: bool = True,
              max_ctas: int = 0):
    """Uneven batched one-launch top-k.

    rows: host list of (in_off, out_off, n, k) or a device uint8/int64 tensor
    holding radik_row_desc records.  Returns flat (vals, idx) of total_out
    slots.  bounds = (total_n, n_max, k_max) for the workspace layout.
    max_ctas > 0 runs the call on at most that many SMs
    (radik_topk_rows_ctas), leaving the others to calls on other streams.
    """
    import torch

    dev = values.device
    if isinstance(rows, torch.Tensor):
        desc = rows
        if bounds is None or total_out is None:
            raise RadikError(EINVAL, "device descriptors need bounds and total_out")
        B = desc.numel() * desc.element_size() // ctypes.sizeof(RowDesc)
    else:
        B = len(rows)
        host = (RowDesc * max(B, 1))()
        for i, (a, b, n, kk) in enumerate(rows):
            host[i] = RowDesc(int(a), int(b), int(n), int(kk))
        raw = torch.frombuffer(bytearray(bytes(host)), dtype=torch.uint8)
        desc = raw.to(dev)
        if bounds is None:
            bounds = (sum(r[2] for r in rows), max((r[2] for r in rows), default=0), max((r[3] for r in rows), default=0))
        if total_out is None:
            total_out = max((r[1] + r[3] for r in rows), default=0)
    total_n, n_max, k_max = bounds
    flags = make_flags(largest, sorted, ascend, with_scale, idx_in is not None, idx64)
    dt = dtype_code(values.dtype)
    _same_device(values, idx_in, workspace, desc)
    with _device_of(values):
        if workspace is None:
            workspace = torch.empty(get_rows_workspace_size(dt, B, total_n, n_max, k_max, flags), dtype=torch.uint8,
                                    device=dev)
        vals = torch.empty(max(total_out, 1), dtype=values.dtype, device=dev)
        idx = torch.empty(max(total_out, 1), dtype=torch.int64 if idx64 else torch.int32, device=dev)
        _check(lib().radik_topk_rows_ctas(dt, flags, values.data_ptr(),
                                          idx_in.data_ptr() if idx_in is not None else None, vals.data_ptr(),
                                          idx.data_ptr(), workspace.data_ptr(), workspace.numel(), desc.data_ptr(), B,
                                          int(total_n), int(n_max), int(k_max), int(max_ctas),
                                          _stream_handle(stream, dev)))
    if check:
        status(workspace, stream)
    return vals[:total_out], idx[:total_out]


STATIC_SCRATCH_BYTES = 32 << 20


def topk_static(values, k: int, lengths: Optional[Sequence[int]] = None, *, largest: bool = True,
                sorted: bool = False, ascend: Optional[bool] = None, with_scale: bool = False, idx_in=None,
                idx64: bool = False, out=None, stream=None, check: bool = True):
    """radik_topk_static: topk() on the library's fixed 32 MiB device scratch.

    The C call allocates nothing.  To keep this wrapper allocation-free too,
    pass ``out=(vals, idx)``: contiguous tensors on the values' device with at
    least B*k elements each, vals of the values' dtype, idx int64 when
    ``idx64`` else int32.  ``values`` (and ``idx_in``) must then be
    contiguous: a strided input would need a copy, so it is rejected rather
    than copied.  Calls that need more scratch raise RadikError(EWORKSPACE).
    Calls in flight at the same time on one device share the scratch and
    must not overlap.
    """
    import torch

    if values.dim() == 2:
        B, n = values.shape
        lengths = [n] * B
    else:
        if lengths is None:
            lengths = [values.numel()]
        B = len(lengths)
    if out is not None:
        if not values.is_contiguous() or (idx_in is not None and not idx_in.is_contiguous()):
            raise RadikError(EINVAL, "topk_static with out=: values and idx_in must be contiguous (a copy would "
                                     "allocate)")
        vals, idx = out
        want_idx = torch.int64 if idx64 else torch.int32
        for name, t, dt_ in (("vals", vals, values.dtype), ("idx", idx, want_idx)):
            if t.dtype != dt_:
                raise RadikError(EINVAL, f"topk_static out {name}: dtype {t.dtype}, expected {dt_}")
            if t.device != values.device:
                raise RadikError(EINVAL, f"topk_static out {name}: on {t.device}, values on {values.device}")
            if not t.is_contiguous():
                raise RadikError(EINVAL, f"topk_static out {name}: must be contiguous")
            if t.numel() < B * k:
                raise RadikError(EINVAL, f"topk_static out {name}: {t.numel()} elements, need {B * k}")
        flat = values
    else:
        flat = values.contiguous()
    _same_device(values, idx_in)
    flags = make_flags(largest, sorted, ascend, with_scale, idx_in is not None, idx64)
    arr = (ctypes.c_int * max(B, 1))(*[int(x) for x in lengths])
    scratch = ctypes.c_void_p(0)
    with _device_of(values):
        if out is None:
            out = (torch.empty((B, k), dtype=values.dtype, device=values.device),
                   torch.empty((B, k), dtype=torch.int64 if idx64 else torch.int32, device=values.device))
        vals, idx = out
        sh = _stream_handle(stream, values.device)
        _check(lib().radik_topk_static(dtype_code(values.dtype), flags, flat.data_ptr(),
                                       idx_in.data_ptr() if idx_in is not None else None, vals.data_ptr(),
                                       idx.data_ptr(), arr, B, int(k), sh, ctypes.byref(scratch)))
        if check and scratch.value:
            bits = ctypes.c_int(0)
            _check(lib().radik_get_status(scratch, sh, ctypes.byref(bits)))
    return vals, idx


# ---------------------------------------------------------------------------
# Serving: continuous-batching request loop (radik_server_* in the C ABI)
# ---------------------------------------------------------------------------
class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("mode", ctypes.c_int), ("slots", ctypes.c_int),
                ("max_batch_rows", ctypes.c_int), ("max_batch_keys", ctypes.c_int64), ("max_n", ctypes.c_int),
                ("max_k", ctypes.c_int), ("budget_bytes", ctypes.c_size_t)]


class Completion(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("latency_us", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_int64), ("requests", ctypes.c_int64), ("batches_beside_others", ctypes.c_int64),
                ("max_batches_in_flight", ctypes.c_int32), ("max_ctas_in_flight", ctypes.c_int32),
                ("ctas_total", ctypes.c_int32), ("ctas_cap", ctypes.c_int32)]


class TraceItem(ctypes.Structure):
    _fields_ = [("arrival_us", ctypes.c_double), ("dtype", ctypes.c_int), ("flags", ctypes.c_uint32),
                ("values", ctypes.c_void_p), ("n", ctypes.c_int), ("k", ctypes.c_int),
                ("val_out", ctypes.c_void_p), ("idx_out", ctypes.c_void_p)]


def _server_lib():
    L = lib()
    if not getattr(L, "_server_bound", False):
        vp = ctypes.c_void_p
        L.radik_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.radik_server_submit.argtypes = [vp, ctypes.c_int, ctypes.c_uint32, vp, ctypes.c_int, ctypes.c_int, vp, vp,
                                          ctypes.POINTER(ctypes.c_uint64)]
        L.radik_server_poll.argtypes = [vp, ctypes.POINTER(Completion), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.radik_server_drain.argtypes = [vp]
        L.radik_server_run_trace.argtypes = [vp, ctypes.POINTER(TraceItem), ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.radik_server_destroy.argtypes = [vp]
        L.radik_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        for name in ("radik_server_create", "radik_server_submit", "radik_server_poll", "radik_server_drain",
                     "radik_server_run_trace", "radik_server_destroy", "radik_server_get_stats"):
            getattr(L, name).restype = ctypes.c_int
        L._server_bound = True
    return L


class Server:
    """Continuous-batching top-k server on one device (radik_server_*).

    mode 0 batches queued requests into one-launch radik_topk_rows calls;
    mode 1 is the per-request baseline (one radik_topk launch each).  Request
    values and result buffers are device tensors owned by the caller and must
    stay alive until the request completes.
    """

    def __init__(self, device: int = 0, mode: int = 0, slots: int = 0, max_batch_rows: int = 0,
                 max_batch_keys: int = 0, max_n: int = 0, max_k: int = 0, budget_bytes: int = 0):
        self._L = _server_lib()
        cfg = ServerConfig(device, mode, slots, max_batch_rows, max_batch_keys, max_n, max_k, budget_bytes)
        h = ctypes.c_void_p(0)
        _check(self._L.radik_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def submit(self, values, k: int, val_out, idx_out, *, largest: bool = True, sorted: bool = False,
               ascend: Optional[bool] = None) -> int:
        flags = make_flags(largest, sorted, ascend, False, False, idx_out.dtype.itemsize == 8)
        rid = ctypes.c_uint64(0)
        _check(self._L.radik_server_submit(self._h, dtype_code(values.dtype), flags, values.data_ptr(),
                                           int(values.numel()), int(k), val_out.data_ptr(), idx_out.data_ptr(),
                                           ctypes.byref(rid)))
        return rid.value

    def poll(self, max_items: int = 4096):
        buf = (Completion * max_items)()
        cnt = ctypes.c_int(0)
        _check(self._L.radik_server_poll(self._h, buf, max_items, ctypes.byref(cnt)))
        return [(buf[i].id, buf[i].status, buf[i].latency_us) for i in range(cnt.value)]

    def drain(self) -> None:
        _check(self._L.radik_server_drain(self._h))

    def stats(self) -> dict:
        """The server's batch counters (radik_server_get_stats)."""
        st = ServerStats()
        _check(self._L.radik_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def run_trace(self, items) -> "list":
        """items: sequence of TraceItem; returns per-item latencies (us)."""
        arr = (TraceItem * max(len(items), 1))(*items)
        lat = (ctypes.c_double * max(len(items), 1))()
        _check(self._L.radik_server_run_trace(self._h, arr, len(items), lat))
        return list(lat)[:len(items)]

    def close(self) -> None:
        if self._h:
            self._L.radik_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(values, k: int, lengths: Optional[Sequence[int]] = None, *, largest: bool = True, sorted: bool = False,
             workspace=None, stream=None) -> dict:
    """radik_autotune_ex: times the knobs of this call's shape bucket (dtype,
    sortedness, log2 of rows, longest row, k) on these buffers -- the chunk
    length, the first-digit width and the one-CTA row cap -- and keeps the
    fastest for later calls in this process.  Returns the choice as a dict
    (0: the built-in value).  Synchronises ``stream``."""
    import torch

    if values.dim() == 2:
        B, n = values.shape
        lengths = [n] * B
        flat = values.contiguous().view(-1)
    else:
        lengths = list(lengths) if lengths is not None else [values.numel()]
        flat = values.contiguous()
        B = len(lengths)
    flags = make_flags(largest, sorted)
    dt = dtype_code(values.dtype)
    _same_device(values, workspace)
    with _device_of(values):
        if workspace is None:
            workspace = torch.empty(get_radix_select_l_workspace_size(dt, k, max(lengths), B, flags),
                                    dtype=torch.uint8, device=values.device)
        vals = torch.empty((B, k), dtype=values.dtype, device=values.device)
        idx = torch.empty((B, k), dtype=torch.int32, device=values.device)
        arr = (ctypes.c_int * max(B, 1))(*[int(x) for x in lengths])
        choice = TuneChoice()
        _check(lib().radik_autotune_ex(dt, flags, flat.data_ptr(), None, vals.data_ptr(), idx.data_ptr(),
                                       workspace.data_ptr(), workspace.numel(), arr, B, int(k),
                                       _stream_handle(stream, values.device), ctypes.byref(choice)))
    return choice.as_dict()


def autotune_rows(values, desc, B: int, bounds: Tuple[int, int, int], total_out: int, *, largest: bool = True,
                  sorted: bool = False, workspace=None, stream=None) -> dict:
    """radik_autotune_rows: the engine's knobs for a radik_topk_rows call
    (device descriptors ``desc``; bounds = (total_n, n_max, k_max))."""
    import torch

    total_n, n_max, k_max = bounds
    flags = make_flags(largest, sorted)
    dt = dtype_code(values.dtype)
    with _device_of(values):
        if workspace is None:
            workspace = torch.empty(get_rows_workspace_size(dt, B, total_n, n_max, k_max, flags), dtype=torch.uint8,
                                    device=values.device)
        vals = torch.empty(max(total_out, 1), dtype=values.dtype, device=values.device)
        idx = torch.empty(max(total_out, 1), dtype=torch.int32, device=values.device)
        choice = TuneChoice()
        _check(lib().radik_autotune_rows(dt, flags, values.data_ptr(), None, vals.data_ptr(), idx.data_ptr(),
                                         workspace.data_ptr(), workspace.numel(), desc.data_ptr(), B, int(total_n),
                                         int(n_max), int(k_max), _stream_handle(stream, values.device),
                                         ctypes.byref(choice)))
    return choice.as_dict()


def autotune_save(path: str) -> None:
    """Writes the tuned buckets to a text file (RADIK_TUNE_FILE loads it)."""
    _check(lib().radik_autotune_save(os.fsencode(path)))


def autotune_load(path: str) -> None:
    """Replaces the tuned buckets with a file's."""
    _check(lib().radik_autotune_load(os.fsencode(path)))


def autotune_reset() -> None:
    lib().radik_autotune_reset()
