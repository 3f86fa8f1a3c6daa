"""radik_topk_static (fixed device scratch, no allocation) against radik_topk
(caller-owned workspace) on the same inputs.  Kept in a file collected last so
that it also runs after every other GPU test has used the device."""
import numpy as np
import pytest

from radik_b200 import workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import radik_b200 as rk  # noqa: E402

DEV = "cuda:0"


def _by_index(v, i):
    """(values, indices) of each row ordered by index, for unsorted outputs."""
    order = torch.argsort(i.to(torch.int64), dim=1)
    return torch.gather(v, 1, order), torch.gather(i, 1, order)


def test_two_calls_in_a_row_match_workspace_entry_point():
    # call 1: pre-filter rows, unsorted; call 2: one-CTA rows, sorted, f16
    x1 = torch.from_numpy(workloads.normal(8 << 20, 31)).to(DEV).view(8, 1 << 20)
    x2 = torch.from_numpy(workloads.uniform01(64 * 100000, 32).astype(np.float16)).to(DEV).view(64, 100000)
    s1 = rk.topk_static(x1, 256, largest=True, sorted=False)
    s2 = rk.topk_static(x2, 1000, largest=False, sorted=True)
    w1 = rk.topk(x1, 256, largest=True, sorted=False)
    w2 = rk.topk(x2, 1000, largest=False, sorted=True)
    a, b = _by_index(*s1), _by_index(*w1)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert torch.equal(s2[0], w2[0]) and torch.equal(s2[1], w2[1])
    # and again on the scratch the previous calls left behind
    s1b = rk.topk_static(x1, 256, largest=True, sorted=True)
    w1b = rk.topk(x1, 256, largest=True, sorted=True)
    assert torch.equal(s1b[0], w1b[0]) and torch.equal(s1b[1], w1b[1])


def test_uneven_lengths_through_the_static_scratch():
    # rows of unequal length take the planning kernel, whose descriptors the
    # call copies into the static scratch too
    lengths = [100003, 5, 70000, 1 << 20, 16385, 3000]
    x = torch.from_numpy(workloads.normal(sum(lengths), 33)).to(DEV)
    for sorted_ in (False, True):
        s = rk.topk_static(x, 300, lengths, largest=True, sorted=sorted_)
        w = rk.topk(x, 300, lengths, largest=True, sorted=sorted_)
        if not sorted_:
            s, w = _by_index(*s), _by_index(*w)
        assert torch.equal(s[0], w[0]) and torch.equal(s[1], w[1])


def test_a_call_allocates_no_device_memory():
    """With out= given, a call after the first one on the device changes
    neither the driver's free-memory figure nor torch's allocator."""
    x = torch.from_numpy(workloads.normal(4 << 20, 34)).to(DEV).view(4, 1 << 20)
    vals = torch.empty((4, 128), dtype=torch.float32, device=DEV)
    idx = torch.empty((4, 128), dtype=torch.int32, device=DEV)
    rk.topk_static(x, 128, out=(vals, idx), sorted=True)  # first call on the device: symbol lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    rk.topk_static(x, 128, out=(vals, idx), sorted=True, check=False)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 == free0
    w = rk.topk(x, 128, sorted=True)
    assert torch.equal(vals, w[0]) and torch.equal(idx, w[1])


def test_out_buffers_are_validated():
    x = torch.zeros((2, 4096), dtype=torch.float32, device=DEV)
    good_v = torch.empty((2, 16), dtype=torch.float32, device=DEV)
    good_i = torch.empty((2, 16), dtype=torch.int32, device=DEV)
    bad = [(torch.empty(31, dtype=torch.float32, device=DEV), good_i),          # too short
           (good_v, torch.empty((2, 16), dtype=torch.int64, device=DEV)),       # idx dtype
           (good_v.half(), good_i),                                             # value dtype
           (torch.empty((16, 2), dtype=torch.float32, device=DEV).t(), good_i)]  # not contiguous
    for out in bad:
        with pytest.raises(rk.RadikError) as err:
            rk.topk_static(x, 16, out=out)
        assert err.value.code == rk.EINVAL
    with pytest.raises(rk.RadikError):
        rk.topk_static(torch.zeros((4096, 2), device=DEV).t(), 16, out=(good_v, good_i))


def test_call_beyond_the_static_scratch_is_rejected():
    B, n, k = 40, 1 << 20, 256
    need = rk.get_radix_select_l_workspace_size(rk.F32, k, n, B, 0)
    assert need > rk.STATIC_SCRATCH_BYTES
    x = torch.zeros((B, n), dtype=torch.float32, device=DEV)
    with pytest.raises(rk.RadikError) as err:
        rk.topk_static(x, k, largest=True, sorted=False)
    assert err.value.code == rk.EWORKSPACE
    assert "static" in str(err.value) and str(rk.STATIC_SCRATCH_BYTES) in str(err.value)
    # the message states this call's own need
    assert " need " in str(err.value)
