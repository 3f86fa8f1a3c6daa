"""Seeded synthetic inputs for the benchmark shapes and the parity tests.

All randomness comes from numpy's Philox-4x32-10 counter-based generator
(Salmon et al., SC'11), so every host produces the same bits for the same
seed.  These stand in for the reference's benchmark data (cuRAND U(0,1) and
the std::default_random_engine fixtures of radik/test/test_radik.cu:89-121,
and the Zipf sampler of radik/test/zipf.hpp).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def uniform01(n: int, seed: int) -> np.ndarray:
    """fp32 U[0,1): 24 random bits times 2^-24 (numpy's float32 draw)."""
    return rng(seed).random(n, dtype=np.float32)


def uniform_rows(B: int, n: int, seed: int) -> np.ndarray:
    """B rows of n U(0,1) values, row r drawn from seed + r; shape (B, n)."""
    out = np.empty((B, n), dtype=np.float32)
    for r in range(B):
        out[r] = uniform01(n, seed + r)
    return out


def normal(n: int, seed: int) -> np.ndarray:
    return rng(seed).standard_normal(n, dtype=np.float32)


def mantissa_noise(n: int, seed: int) -> np.ndarray:
    """1.0f with random low 8 mantissa bits: every key shares its top 24 bits."""
    r8 = rng(seed).integers(0, 256, n, dtype=np.uint32)
    return (np.uint32(0x3F800000) | r8).view(np.float32)


def zipf_ranks(n: int, s: float, seed: int, n_max: int = None) -> np.ndarray:
    """Zipf(s) integer ranks in [1, n_max] cast to fp32 (no 1/n scaling).

    Rejection sampling (the method radik/test/zipf.hpp follows, restated and
    vectorised): draw x from the continuous density x^-s on [1, n_max+1) by
    inversion, accept with probability (x / floor(x))^s / 2^s, return
    floor(x).  The accepted floor(x) has P(k) proportional to k^-s.
    """
    n_max = n_max or n
    g = rng(seed)
    out = np.empty(n, dtype=np.float32)
    filled = 0
    a = 1.0 - s
    hi = (n_max + 1.0) ** a
    while filled < n:
        m = max(1024, int((n - filled) * 2.2))
        u = g.random(m)
        x = (1.0 + u * (hi - 1.0)) ** (1.0 / a)
        kx = np.minimum(np.floor(x), n_max)
        acc = g.random(m) < (x / kx) ** s / 2.0 ** s
        take = kx[acc][: n - filled]
        out[filled: filled + take.size] = take.astype(np.float32)
        filled += take.size
    return out


def constant_heavy(n: int, seed: int, frac_const: float = 0.9, const: float = 0.5) -> np.ndarray:
    """frac_const of the entries equal to `const`, the rest U(0,1) at random positions."""
    g = rng(seed)
    out = g.random(n, dtype=np.float32)
    mask = g.random(n) < frac_const
    out[mask] = np.float32(const)
    return out


SKEW_DISTRIBUTIONS = ("uniform", "mantissa_noise", "zipf", "constant_heavy")


def skew_row(dist: str, n: int, seed: int) -> np.ndarray:
    if dist == "uniform":
        return uniform01(n, seed)
    if dist == "mantissa_noise":
        return mantissa_noise(n, seed)
    if dist == "zipf":
        return zipf_ranks(n, 1.1, seed)
    if dist == "constant_heavy":
        return constant_heavy(n, seed)
    raise ValueError(dist)


def uneven_rows(B: int, seed: int, log2_lo: int = 10, log2_hi: int = 22, k_cap: int = 2048) -> Tuple[List[int], List[int]]:
    """Row lengths log-uniform in [2^lo, 2^hi], k log-uniform in [1, min(k_cap, n)]."""
    g = rng(seed)
    u = g.random(B)
    n = np.floor(2.0 ** (log2_lo + (log2_hi - log2_lo) * u)).astype(np.int64)
    u2 = g.random(B)
    kmax = np.minimum(k_cap, n)
    k = np.maximum(1, np.floor(np.exp(u2 * np.log(kmax.astype(np.float64))))).astype(np.int64)
    return [int(x) for x in n], [int(x) for x in k]


def uneven_device_values(total_n: int, seed: int, device):
    """N(0,1) fp32 values for the uneven batch, generated on the device with
    torch's Philox generator (seeded, deterministic for a given torch build):
    an 8 GB batch is drawn in milliseconds instead of minutes on the host.
    Drawn in 2^28-value pieces so every call size stays far below 2^31."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty(total_n, dtype=torch.float32, device=device)
    piece = 1 << 28
    for a in range(0, total_n, piece):
        b = min(total_n, a + piece)
        out[a:b] = torch.randn(b - a, generator=g, device=device, dtype=torch.float32)
    return out


def to_f16(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest fp16 of fp32 draws."""
    return x.astype(np.float16)


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even bf16 bit patterns (uint16) of fp32 values."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    nan = np.isnan(x)
    r = ((u + rounding) >> 16).astype(np.uint16)
    r[nan] = 0x7FC0
    return r


def log2_floor(x: int) -> int:
    return int(math.floor(math.log2(x))) if x > 0 else 0
