"""The timeline build (libradik_b200_timeline.so, RADIK_TIMELINE): the normal
library refuses to attach a stamp buffer; the timeline library selects
exactly as the normal one and stamps its phases in order."""
import ctypes
import os

import numpy as np
import pytest

import radik_b200 as rk
from radik_b200 import build

import oracle  # noqa: E402
from conftest import bits_of  # noqa: E402


def test_normal_library_refuses_the_timeline():
    assert rk.lib().radik_timeline_attach(None) == rk.ENOTSUP


def test_timeline_library_exports_the_abi():
    if not os.path.exists(build.LIB_TIMELINE):
        pytest.skip("timeline build not present")
    L = ctypes.CDLL(build.LIB_TIMELINE)
    for name in ("radik_topk", "radik_get_workspace_size", "radik_timeline_attach", "radik_get_status"):
        assert hasattr(L, name)


@pytest.mark.gpu
def test_timeline_library_selects_exactly_and_stamps_in_order():
    import torch

    L = ctypes.CDLL(build.LIB_TIMELINE)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    L.radik_get_workspace_size.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(sz)]
    L.radik_topk.argtypes = [ctypes.c_int, ctypes.c_uint32, vp, vp, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_int),
                             ctypes.c_int, ctypes.c_int, vp]
    L.radik_timeline_attach.argtypes = [vp]
    L.radik_get_status.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int)]
    dev = torch.device("cuda:0")
    n, k = 1 << 20, 256
    host = np.random.default_rng(3).random(n, dtype=np.float32)
    x = torch.from_numpy(host).to(dev)
    need = sz(0)
    assert L.radik_get_workspace_size(rk.F32, rk.LARGEST, k, n, 1, ctypes.byref(need)) == 0
    ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    vals = torch.empty(k, dtype=torch.float32, device=dev)
    idx = torch.empty(k, dtype=torch.int32, device=dev)
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    stamps = torch.zeros(sm * 32, dtype=torch.int64, device=dev)
    lens = (ctypes.c_int * 1)(n)
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert L.radik_timeline_attach(ctypes.c_void_p(stamps.data_ptr())) == 0
    try:
        rc = L.radik_topk(rk.F32, rk.LARGEST, x.data_ptr(), None, vals.data_ptr(), idx.data_ptr(), ws.data_ptr(),
                          ws.numel(), lens, 1, k, ctypes.c_void_p(stream))
        torch.cuda.synchronize(dev)
    finally:
        L.radik_timeline_attach(None)
    assert rc == 0
    bits = ctypes.c_int(-1)
    assert L.radik_get_status(ws.data_ptr(), ctypes.c_void_p(stream), ctypes.byref(bits)) == 0 and bits.value == 0
    ov, oi = oracle.topk(host, [n], k, flags=oracle.flags_of(True, False))
    gi = idx.cpu().numpy()
    order = np.argsort(gi)
    assert np.array_equal(gi[order], np.sort(oi))
    assert np.array_equal(bits_of(vals.cpu().numpy())[order], bits_of(host[np.sort(oi)]))
    t = stamps.view(sm, 32).cpu().numpy()
    ran = t[t[:, 0] > 0]
    assert ran.shape[0] == sm
    assert np.all(ran[:, 6] >= ran[:, 0])  # every CTA's end follows its start
    fin = ran[ran[:, 7] > 0]
    assert fin.shape[0] == 1  # one row, one finish
    assert fin[0, 0] <= fin[0, 7] <= fin[0, 16] <= fin[0, 17] <= fin[0, 18] <= fin[0, 19] <= fin[0, 4] <= fin[0, 6]
    assert 0 < fin[0, 31] <= n  # candidate count
