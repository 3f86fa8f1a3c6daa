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


def test_call_beyond_the_static_scratch_is_rejected():
    B, n, k = 40, 1 << 20, 256
    need = rk.get_radix_select_l_workspace_size(rk.F32, k, n, B, 0)
    assert need > rk.STATIC_SCRATCH_BYTES
    x = torch.zeros((B, n), dtype=torch.float32, device=DEV)
    with pytest.raises(rk.RadikError) as err:
        rk.topk_static(x, k, largest=True, sorted=False)
    assert err.value.code == rk.EWORKSPACE
    assert "static" in str(err.value) and str(rk.STATIC_SCRATCH_BYTES) in str(err.value)
