"""Generates the golden fixtures that pin the oracle to the reference RadiK.

Runs the UNMODIFIED reference RadiK (oracle/_ref/libradik_ref.so, compiled
from the reference's own sources by oracle/Makefile) on a CUDA device over
small seeded inputs and saves inputs + RadiK's outputs as .npz files.
tests/test_oracle.py then checks the CPU oracle against them with no GPU.

Usage (on a machine with a B200):  python tests/golden/make_golden.py OUTDIR
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from radik_b200 import workloads  # noqa: E402

# name, dtype, lengths, K, largest, ascend, withscale, sorted, distribution, seed
# (no row shorter than K: the reference launches a zero-sized grid for it and
# raises "invalid configuration argument", topk_radixselect.h:158-168)
CASES = [
    ("f32_u01_largest_unsorted", oracle.F32, [3000] * 4, 32, 1, 0, 0, 0, "u01", 1),
    ("f32_u01_largest_sorted_multichunk", oracle.F32, [70000], 256, 1, 0, 0, 1, "u01", 2),
    ("f32_normal_smallest_sorted", oracle.F32, [5000] * 3, 100, 0, 1, 0, 1, "normal", 3),
    ("f16_u01_largest_sorted", oracle.F16, [4000] * 4, 64, 1, 0, 0, 1, "u01", 4),
    ("f32_u0607_scaled_largest_sorted", oracle.F32, [20000] * 2, 1024, 1, 0, 1, 1, "u0607", 5),
    ("f16_u0607_scaled_smallest_unsorted", oracle.F16, [6000] * 2, 77, 0, 1, 1, 0, "u0607", 6),
    ("f32_all_zero_unsorted", oracle.F32, [5000], 50, 1, 0, 0, 0, "zero", 8),
    ("f32_uneven_lengths_sorted", oracle.F32, [7400, 8800, 8000, 7300, 8700], 128, 0, 1, 0, 1, "u01", 9),
    ("f32_u12867_largest_unsorted", oracle.F32, [40000], 500, 1, 0, 0, 0, "u128", 10),
]


def make(dist, n, seed):
    g = workloads.rng(seed)
    if dist == "u01":
        return workloads.uniform01(n, seed)
    if dist == "normal":
        return workloads.normal(n, seed)
    if dist == "u0607":
        return (np.float32(0.6) + np.float32(0.1) * g.random(n, dtype=np.float32)).astype(np.float32)
    if dist == "u128":
        return (np.float32(128.6) + np.float32(0.1) * g.random(n, dtype=np.float32)).astype(np.float32)
    if dist == "zero":
        return np.zeros(n, dtype=np.float32)
    raise ValueError(dist)


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    ref = oracle.RefRadik()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for name, dtype, lengths, K, largest, ascend, scale, srt, dist, seed in CASES:
        rows = [make(dist, n, seed * 1000 + r) for r, n in enumerate(lengths)]
        vals = np.concatenate(rows)
        if dtype == oracle.F16:
            vals = vals.astype(np.float16)
        B = len(lengths)
        tin = torch.from_numpy(vals).to(dev)
        vout = torch.zeros(B * K, dtype=tin.dtype, device=dev)
        iout = torch.zeros(B * K, dtype=torch.int32, device=dev)
        ws = torch.zeros(ref.workspace_size(dtype, K, max(lengths), B), dtype=torch.uint8, device=dev)
        ref.topk(dtype, largest, ascend, scale, srt, tin.data_ptr(), vout.data_ptr(), iout.data_ptr(),
                 ws.data_ptr(), lengths, K, stream)
        torch.cuda.synchronize()
        flags = oracle.flags_of(bool(largest), bool(srt), bool(ascend), bool(scale))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), values=vals, lengths=np.array(lengths),
                            K=K, dtype=dtype, flags=flags, ref_vals=vout.cpu().numpy(), ref_idx=iout.cpu().numpy())
        print("wrote", name, flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
