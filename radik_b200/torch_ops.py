"""PyTorch operator over the C ABI: ``torch.ops.radik.topk``.

    vals, idx = torch.ops.radik.topk(values, k, lengths, largest, sorted)

``values`` is a CUDA tensor (fp32 / fp16 / bf16): 2-D rows of equal length, or
1-D rows back to back with ``lengths`` (a list of row lengths; empty list = one
row, or the rows of a 2-D input).  Returns ``vals [B, k]`` and ``idx [B, k]``
(int64, positions within each row; slots past a short row hold -1 / 0).  The
selection is exact with ties at the k-th value going to the lowest positions,
so for distinct values it returns the same sets as ``torch.topk``.

Importing this module registers the operator (and a shape function, so the op
traces under ``torch.compile`` / fake tensors).  The compute always runs in
libradik_b200.so; there is no fallback.
"""
from __future__ import annotations

from typing import List, Tuple

import torch

import radik_b200 as _rk


@torch.library.custom_op("radik::topk", mutates_args=())
def topk(values: torch.Tensor, k: int, lengths: List[int], largest: bool = True,
         sorted: bool = True) -> Tuple[torch.Tensor, torch.Tensor]:
    if not values.is_cuda:
        raise ValueError("radik::topk needs a CUDA tensor (there is no CPU implementation)")
    if values.dim() == 2:
        vals, idx = _rk.topk(values, int(k), None, largest=largest, sorted=sorted, idx64=True)
    else:
        lens = list(lengths) if len(lengths) else [values.numel()]
        vals, idx = _rk.topk(values, int(k), lens, largest=largest, sorted=sorted, idx64=True)
    return vals, idx


@topk.register_fake
def _(values, k, lengths, largest=True, sorted=True):
    B = values.shape[0] if values.dim() == 2 else max(len(lengths), 1)
    return (values.new_empty((B, k)), values.new_empty((B, k), dtype=torch.int64))
