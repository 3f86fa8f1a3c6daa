"""torch.ops.radik.topk: registration and shapes on CPU (fake tensors), and on
the GPU against torch.topk as a second reference (distinct values, so the
index sets are unique)."""
import pytest

torch = pytest.importorskip("torch")

import radik_b200.torch_ops  # noqa: E402,F401  (registers radik::topk)


def test_op_registered_with_shape_function():
    from torch._subclasses.fake_tensor import FakeTensorMode

    with FakeTensorMode():
        x = torch.empty(4, 100, device="cuda")
        v, i = torch.ops.radik.topk(x, 7, [], True, True)
        assert tuple(v.shape) == (4, 7) and tuple(i.shape) == (4, 7) and i.dtype == torch.int64
        y = torch.empty(300, device="cuda", dtype=torch.float16)
        v, i = torch.ops.radik.topk(y, 5, [100, 200], False, False)
        assert tuple(v.shape) == (2, 5) and v.dtype == torch.float16


def test_cpu_tensor_is_rejected():
    with pytest.raises(ValueError):
        torch.ops.radik.topk(torch.randn(10), 3, [], True, True)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("largest", [True, False])
@pytest.mark.parametrize("shape,k", [((8, 1 << 20), 256), ((3, 50000), 1000), ((64, 4096), 17)])
def test_matches_torch_topk(dtype, largest, shape, k):
    g = torch.Generator(device="cuda").manual_seed(5)
    # distinct values: a permutation scaled into the dtype's exact integer range
    B, n = shape
    base = torch.stack([torch.randperm(n, device="cuda", generator=g) for _ in range(B)])
    lim = {torch.float32: 1 << 24, torch.float16: 2048, torch.bfloat16: 256}[dtype]
    if n > lim:
        x = (base.float() / n).to(dtype)  # ties possible: compare values only
        exact_idx = False
    else:
        x = base.to(dtype)
        exact_idx = True
    v, i = torch.ops.radik.topk(x, k, [], largest, True)
    tv, ti = torch.topk(x, k, dim=1, largest=largest, sorted=True)
    assert torch.equal(v, tv)
    assert torch.equal(torch.gather(x, 1, i), v)
    if exact_idx:
        assert torch.equal(i, ti)
