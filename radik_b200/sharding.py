"""Rows across GPUs: one process per GPU, rows split into contiguous ranges.

Rows are independent, so a batch shards with no collective on the data path:
rank r selects the rows of its range on its own GPU and writes its own slice of
the outputs.  ``gather_rows`` is only for callers that want every row's
results on one rank (an ``all_gather`` of the per-rank slices).
"""
from __future__ import annotations

import bisect
from typing import List, Sequence, Tuple


def shard_rows(lengths: Sequence[int], world: int, rank: int) -> Tuple[int, int]:
    """[first, last) row range of ``rank``: contiguous ranges with about equal
    sums of n (the keys each GPU reads); with at least ``world`` rows every
    range is non-empty."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    B = len(lengths)
    prefix = [0]
    for n in lengths:
        prefix.append(prefix[-1] + int(n))
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        target = r * total / world
        i = bisect.bisect_left(prefix, target)
        lo = cuts[-1] + (1 if B >= world else 0)
        hi = B - (world - r) if B >= world else B
        cuts.append(min(max(i, lo), hi))
    cuts.append(B)
    return cuts[rank], cuts[rank + 1]


def shard_bounds(lengths: Sequence[int], world: int) -> List[Tuple[int, int]]:
    return [shard_rows(lengths, world, r) for r in range(world)]


def gather_rows(vals, idx, k: int, lengths: Sequence[int], group=None):
    """All-gathers per-rank (vals [b_r, k], idx [b_r, k]) slices, in rank
    order, into full (vals [B, k], idx [B, k]) on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    bounds = shard_bounds(lengths, world)
    Bmax = max(b - a for a, b in bounds)
    pv = torch.zeros((Bmax, k), dtype=vals.dtype, device=vals.device)
    pi = torch.zeros((Bmax, k), dtype=idx.dtype, device=idx.device)
    pv[: vals.shape[0]] = vals
    pi[: idx.shape[0]] = idx
    gv = [torch.empty_like(pv) for _ in range(world)]
    gi = [torch.empty_like(pi) for _ in range(world)]
    dist.all_gather(gv, pv, group=group)
    dist.all_gather(gi, pi, group=group)
    out_v = torch.cat([g[: b - a] for g, (a, b) in zip(gv, bounds)])
    out_i = torch.cat([g[: b - a] for g, (a, b) in zip(gi, bounds)])
    return out_v, out_i


# ---------------------------------------------------------------------------
# One row split over the ranks
# ---------------------------------------------------------------------------
# RadiK selects each row on one GPU.  A row longer than one GPU's share is
# held as contiguous shards, one per rank (global positions [pos_base,
# pos_base + n) on rank r), and selected with radix levels over the composite
# (selection key << ib | global position) -- the order a single GPU uses, so
# the result equals the single-GPU one bit for bit.  Each level exchanges one
# 4096-counter histogram (an all-reduce of 16 KB); the final exchange gathers
# the certainly-selected keys and the tie set (at most cap keys).

_DIGIT = 12


def index_bits(n: int) -> int:
    b = 1
    while b < 32 and (1 << b) < n:
        b += 1
    return b


def key_bits_of(torch_dtype, with_scale: bool) -> int:
    import torch

    return 32 if (torch_dtype == torch.float32 or with_scale) else 16


class DeviceShard:
    """This rank's shard on its GPU, through radik_shard_histogram /
    radik_shard_collect of the C ABI."""

    def __init__(self, values, pos_base: int, ib: int, largest: bool, with_scale: bool, scaler: float):
        import ctypes

        import torch

        from . import LARGEST, WITHSCALE, _check, _device_of, _stream_handle, dtype_code, lib

        self.t, self.pos_base, self.ib, self.scaler = values.contiguous(), int(pos_base), int(ib), float(scaler)
        self.dt = dtype_code(values.dtype)
        self.flags = (LARGEST if largest else 0) | (WITHSCALE if with_scale else 0)
        self._ct, self._check, self._dev_of, self._sh = ctypes, _check, _device_of, _stream_handle
        L = lib()
        if not getattr(L, "_shard_bound", False):
            vp, i32, i64, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64
            L.radik_shard_histogram.argtypes = [i32, ctypes.c_uint32, vp, i64, i64, i32, u64, i32, i32, ctypes.c_float,
                                                vp, vp]
            L.radik_shard_collect.argtypes = [i32, ctypes.c_uint32, vp, i64, i64, i32, u64, i32, ctypes.c_float, vp,
                                              i32, vp, i32, vp, vp]
            L.radik_shard_histogram.restype = i32
            L.radik_shard_collect.restype = i32
            L._shard_bound = True
        self.L = L
        dev = values.device
        self.hist = torch.empty(1 << _DIGIT, dtype=torch.int32, device=dev)
        self.counts = torch.empty(2, dtype=torch.int32, device=dev)

    def histogram(self, prefix: int, plen: int, d: int):
        import torch

        with self._dev_of(self.t):
            self._check(self.L.radik_shard_histogram(self.dt, self.flags, self.t.data_ptr(), self.t.numel(),
                                                     self.pos_base, self.ib, prefix, plen, d, self.scaler,
                                                     self.hist.data_ptr(), self._sh(None, self.t.device)))
        # counters are below 2^31 (positions fit in ib <= 31 bits)
        return self.hist[: 1 << d].to(torch.int64)

    def collect(self, prefix: int, plen: int, cap_better: int, cap_tied: int):
        import torch

        dev = self.t.device
        better = torch.empty(max(cap_better, 1), dtype=torch.int64, device=dev)
        tied = torch.empty(max(cap_tied, 1), dtype=torch.int64, device=dev)
        with self._dev_of(self.t):
            self._check(self.L.radik_shard_collect(self.dt, self.flags, self.t.data_ptr(), self.t.numel(),
                                                   self.pos_base, self.ib, prefix, plen, self.scaler,
                                                   better.data_ptr(), cap_better, tied.data_ptr(), cap_tied,
                                                   self.counts.data_ptr(), self._sh(None, dev)))
        nb, nt = (int(v) for v in self.counts.cpu().tolist())
        return better[: min(nb, cap_better)], tied[: min(nt, cap_tied)], nb, nt


def _composites(entries, torch_dtype, largest: bool, with_scale: bool, scaler: float, ib: int):
    """(selection key << ib | position) of entries (value bits << 32 |
    position), the order of the library's selection: the order-preserving
    image of the value (negative: all bits flipped, else the sign bit), of
    float(x) - scaler under WITHSCALE, complemented for largest."""
    import torch

    bits = (entries >> 32) & 0xFFFFFFFF
    pos = entries & 0xFFFFFFFF
    kb = key_bits_of(torch_dtype, with_scale)
    if with_scale:
        if torch_dtype == torch.float32:
            x = bits.to(torch.int32).view(torch.float32)
        else:
            x = (bits & 0xFFFF).to(torch.int16).view(torch_dtype).to(torch.float32)
        d = x - torch.tensor(scaler, dtype=torch.float32, device=x.device)
        bits = d.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    if kb == 32:
        neg = (bits >> 31) & 1
        ukey = torch.where(neg == 1, bits ^ 0xFFFFFFFF, bits ^ 0x80000000)
    else:
        bits = bits & 0xFFFF
        neg = (bits >> 15) & 1
        ukey = torch.where(neg == 1, bits ^ 0xFFFF, bits ^ 0x8000)
    key = ukey ^ ((1 << kb) - 1) if largest else ukey
    return (key << ib) | pos


def split_row_select(shards, reduce_sum, gather, n_total: int, k: int, torch_dtype, largest: bool,
                     with_scale: bool = False, scaler: float = 0.0, sorted: bool = False, cap: int = 4096):
    """The exchange protocol over this process's shards.

    shards: objects with histogram(prefix, plen, d) -> int64 counts and
    collect(prefix, plen, cap_better, cap_tied) -> (better, tied, nb, nt)
    entries; reduce_sum(t) sums a local int64 tensor over all ranks;
    gather(t) concatenates a local int64 tensor's entries from all ranks.
    Returns (value bits, global positions) of the min(k, n_total) selected
    keys, ordered by the selection (sorted) or by position."""
    import torch

    kb = key_bits_of(torch_dtype, with_scale)
    ib = index_bits(n_total)
    w = kb + ib
    kk = min(k, n_total)
    prefix, plen, krem, count = 0, 0, kk, n_total
    while count != krem and count > cap and plen < w:
        d = min(_DIGIT, w - plen)
        h = shards[0].histogram(prefix, plen, d)
        for s in shards[1:]:
            h = h + s.histogram(prefix, plen, d)
        h = reduce_sum(h)
        cum = torch.cumsum(h, 0)
        b = int(torch.searchsorted(cum, torch.tensor([krem], dtype=cum.dtype, device=cum.device)).item())
        below = int(cum[b].item() - h[b].item())
        prefix, plen, krem, count = (prefix << d) | b, plen + d, krem - below, int(h[b].item())
    better_l, tied_l = [], []
    for s in shards:
        bt, tt, nb, nt = s.collect(prefix, plen, kk, max(count, 1))
        better_l.append(bt)
        tied_l.append(tt)
    better = gather(torch.cat(better_l))
    tied = gather(torch.cat(tied_l))
    if tied.numel() > krem:
        c = _composites(tied, torch_dtype, largest, with_scale, scaler, ib)
        tied = tied[torch.argsort(c)[:krem]]
    sel = torch.cat([better, tied])
    order = torch.argsort(_composites(sel, torch_dtype, largest, with_scale, scaler, ib)) if sorted else \
        torch.argsort(sel & 0xFFFFFFFF)
    sel = sel[order]
    return (sel >> 32) & 0xFFFFFFFF, sel & 0xFFFFFFFF


def _values_from_bits(bits, torch_dtype):
    import torch

    if torch_dtype == torch.float32:
        return bits.to(torch.int32).view(torch.float32)
    return (bits & 0xFFFF).to(torch.int16).view(torch_dtype)


def topk_split_row(shard, k: int, *, pos_base: int, n_total: int, largest: bool = True, sorted: bool = False,
                   with_scale: bool = False, scaler: float = 0.0, group=None, cap: int = 4096):
    """Top-k of one row whose contiguous shards live on the ranks of
    ``group`` (this rank: ``shard``, global positions [pos_base, pos_base +
    shard.numel())).  Collective: every rank calls it with the same k,
    n_total and flags, and every rank receives the result: (values [k],
    global positions [k], int64), slots past n_total holding value 0 and
    position -1, as the library's idle fill.  With WITHSCALE the caller
    passes the row's first value as ``scaler`` (0 if NaN or infinite)."""
    import torch
    import torch.distributed as dist

    ib = index_bits(n_total)
    ops = DeviceShard(shard, pos_base, ib, largest, with_scale, scaler)
    return _finish_split(split_row_select([ops], lambda t: _all_reduce_sum(t, group), lambda t: _all_gather_cat(t, group),
                                          n_total, k, shard.dtype, largest, with_scale, scaler, sorted, cap),
                         k, shard.dtype, shard.device)


def topk_split_row_local(shards, k: int, *, pos_bases, n_total: int, largest: bool = True, sorted: bool = False,
                         with_scale: bool = False, scaler: float = 0.0, cap: int = 4096):
    """The same protocol with every shard in this process (the exchanges are
    plain sums and concatenations): the split-row path on one GPU."""
    ib = index_bits(n_total)
    ops = [DeviceShard(s, b, ib, largest, with_scale, scaler) for s, b in zip(shards, pos_bases)]
    return _finish_split(split_row_select(ops, lambda t: t, lambda t: t, n_total, k, shards[0].dtype, largest,
                                          with_scale, scaler, sorted, cap), k, shards[0].dtype, shards[0].device)


def _finish_split(sel, k, torch_dtype, device):
    import torch

    bits, pos = sel
    vals = torch.zeros(k, dtype=torch_dtype, device=device)
    idx = torch.full((k,), -1, dtype=torch.int64, device=device)
    m = bits.numel()
    vals[:m] = _values_from_bits(bits, torch_dtype).to(device)
    idx[:m] = pos.to(device)
    return vals, idx


def _all_reduce_sum(t, group):
    import torch.distributed as dist

    t = t.clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def _all_gather_cat(t, group):
    """Concatenation, in rank order, of every rank's 1-D tensor."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    n = torch.tensor([t.numel()], dtype=torch.int64, device=t.device)
    ns = [torch.empty_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    sizes = [int(x.item()) for x in ns]
    mx = max(sizes + [1])
    pad = torch.zeros(mx, dtype=t.dtype, device=t.device)
    pad[: t.numel()] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)])
