#!/usr/bin/env python
"""Benchmark of the radix top-k hot path (one JSON line on rank 0).

Default workload: plain batched top-k, 256 fp32 rows x 2^20 values, k = 256,
largest, unsorted, values i.i.d. U(0,1) (row r from Philox seed r).  One step
is one radik_topk call over the whole batch.  The inputs (1 GiB) are larger
than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl radik_b200|reference]
                  [--workload batched|batched_k32|batched_k1024|batched_f16|single|skew|uneven]

--impl reference runs the reference RadiK (topKRadixSelectL compiled from the
reference's own sources into oracle/_ref/libradik_ref.so) on the same
workload; the reference has no CPU implementation of the path.
Under torchrun every rank runs the workload on its own GPU (rows are
independent; no collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (B, n, k, dtype, sorted, largest, description)
    "batched": (256, 1 << 20, 256, "f32", False, True, "plain batched top-k, 256 fp32 rows x 2^20, k=256, largest, unsorted, U(0,1)"),
    "batched_k32": (256, 1 << 20, 32, "f32", False, True, "plain batched top-k, 256 fp32 rows x 2^20, k=32, largest, unsorted, U(0,1)"),
    "batched_k1024": (256, 1 << 20, 1024, "f32", False, True, "plain batched top-k, 256 fp32 rows x 2^20, k=1024, largest, unsorted, U(0,1)"),
    "batched_sorted": (256, 1 << 20, 256, "f32", True, True, "plain batched top-k, 256 fp32 rows x 2^20, k=256, largest, sorted, U(0,1)"),
    "batched_f16": (256, 1 << 20, 256, "f16", False, True, "plain batched top-k, 256 fp16 rows x 2^20, k=256, largest, unsorted, U(0,1) rounded to fp16"),
    "single": (1, 1 << 20, 256, "f32", False, True, "plain single-row top-k, one fp32 row of 2^20, k=256, largest, unsorted, U(0,1) seed 0"),
}


# DRAM bytes (read + write) per engine launch measured by ncu, for the
# workloads whose capture is summarised under profiles/ (the 256-row figure is
# the 64-row capture scaled by rows: traffic grows with the rows streamed).
NCU_TRAFFIC = {
    ("batched", 256): 4 * (274446592 + 5250048),  # profiles/engine_kernel_f32_64x1M_k256_full.md
    ("batched", 64): 274446592 + 5250048,
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the GPU is busy."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        finally:
            os.unlink(self.path)
        if not rows:
            return None
        sm = [r[0] for r in rows]
        busy = [r for r in rows if r[0] >= 0.5 * max(sm)] or rows
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in busy for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(busy), "reasons": reasons}


def make_inputs(B, n, dtype):
    from radik_b200 import workloads

    x = workloads.uniform_rows(B, n, 0)
    if dtype == "f16":
        x = x.astype(np.float16)
    return x


def cpu_baseline(x: np.ndarray, B, n, k, sorted_, largest, budget_s: float):
    """The oracle (OpenMP nth_element + sort per row) on the host cores."""
    import oracle

    flags = oracle.flags_of(largest, sorted_)
    flat = x.reshape(-1)
    rows = B
    # bounded sample: whole rows, as many as fit about budget_s of CPU time
    t0 = time.perf_counter()
    oracle.topk(flat[: n], [n], k, flags=flags)
    one = max(time.perf_counter() - t0, 1e-4)
    threads = oracle.max_threads()
    est_rows = int(budget_s / one * max(1, threads) * 0.5)
    rows = max(1, min(B, est_rows))
    sample = flat[: rows * n]
    reps = 0
    t0 = time.perf_counter()
    while True:
        oracle.topk(sample, [n] * rows, k, flags=flags)
        reps += 1
        if time.perf_counter() - t0 > min(budget_s, 30.0) or reps >= 50:
            break
    dt = time.perf_counter() - t0
    keys = reps * rows * n
    return {"value": round(keys / dt / 1e9, 4), "unit": "Gkeys/s", "cores": threads, "kind": "port",
            "sample": f"{reps} x {rows} rows of the workload ({rows * n} keys per pass), OpenMP nth_element"
                      f"{' + sort' if sorted_ else ''} per row on {threads} host threads"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="radik_b200", choices=["radik_b200", "reference"])
    ap.add_argument("--workload", default="batched", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows", type=int, default=0, help="override the row count (profiling a smaller case)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # rank 0 alone times the reference; the other ranks exit without work
        if rank != 0:
            return
        world = 1
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    B, n, k, dts, sorted_, largest, desc = WORKLOADS[args.workload]
    if args.rows > 0:
        B = args.rows
        desc = desc.replace("256 ", f"{B} ", 1)

    x = make_inputs(B, n, dts)
    tdtype = torch.float16 if dts == "f16" else torch.float32
    es = 2 if dts == "f16" else 4
    host = torch.from_numpy(x.reshape(-1)).pin_memory()
    dev_in = host.to(dev)
    vals = torch.empty(B * k, dtype=tdtype, device=dev)
    idx = torch.empty(B * k, dtype=torch.int32, device=dev)
    vals_h = torch.empty(B * k, dtype=tdtype).pin_memory()
    idx_h = torch.empty(B * k, dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream(dev)
    lengths = [n] * B

    if args.impl == "reference":
        import oracle

        ref = oracle.RefRadik()
        dcode = 1 if dts == "f16" else 0
        ws = torch.empty(ref.workspace_size(dcode, k, n, B), dtype=torch.uint8, device=dev)

        def step(inp):
            ref.topk(dcode, largest, not largest, False, sorted_, inp.data_ptr(), vals.data_ptr(), idx.data_ptr(),
                     ws.data_ptr(), lengths, k, stream.cuda_stream)
        launches_per_step = None
    else:
        import radik_b200 as rk

        dcode = rk.F16 if dts == "f16" else rk.F32
        flags = rk.make_flags(largest, sorted_)
        ws = torch.empty(rk.get_radix_select_l_workspace_size(dcode, k, n, B, flags), dtype=torch.uint8, device=dev)

        def step(inp):
            rk.topk_radix_select_l(inp, None, vals, idx, ws, lengths, k, largest=largest, ascend=not largest,
                                   need_sorting=sorted_, stream=stream)
        launches_per_step = 1  # the selection engine (uniform rows need no planning kernel)

    for _ in range(args.warmup):
        step(dev_in)
    torch.cuda.synchronize(dev)
    if args.impl != "reference":
        import radik_b200 as rk

        rk.status(ws, stream)

    sampler = ClockSampler(dev.index)
    sampler.start()
    time.sleep(0.3)
    # ---- device-timed region: inputs resident in HBM
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        evs[i][0].record(stream)
        step(dev_in)
        evs[i][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    total_ms = t_start.elapsed_time(t_end)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    # ---- end-to-end: host buffers, copies inside the timed region
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for i in range(args.steps):
        dev_in.copy_(host, non_blocking=True)
        step(dev_in)
        vals_h.copy_(vals, non_blocking=True)
        idx_h.copy_(idx, non_blocking=True)
    e_end.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e_start.elapsed_time(e_end)
    clocks = sampler.stop()
    if args.impl != "reference":
        rk.status(ws, stream)

    if world > 1:
        t = torch.tensor([total_ms, e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_ms = float(t[0]), float(t[1])

    keys_per_step = B * n
    ms_per_step = total_ms / args.steps
    value = world * keys_per_step * args.steps / (total_ms / 1e3) / 1e9
    e2e_value = world * keys_per_step * args.steps / (e2e_ms / 1e3) / 1e9
    algo_bytes = keys_per_step * es + B * k * (es + 4)
    peak, peak_kind = load_peaks()
    avg_step_s = statistics.mean(step_ms) / 1e3
    achieved = algo_bytes / avg_step_s / 1e9

    out = {
        "metric": "Gkeys/s & % HBM peak; uneven-batch speedup vs plain per-row; serving p50/p99",
        "value": round(value, 3),
        "unit": "Gkeys/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": dts,
        "data": "synthetic: U(0,1) from numpy Philox-4x32-10, row r seed r",
        "config": {"workload": desc, "rows": B, "n": n, "k": k, "sorted": sorted_, "largest": largest,
                   "l2": "inputs (%d MiB) larger than L2; no flush" % (keys_per_step * es >> 20),
                   "parallelism": f"rows replicated per GPU x{world} (no collective)"},
        "e2e": {"value": round(e2e_value, 3), "unit": "Gkeys/s", "h2d_bytes_per_step": keys_per_step * es,
                "d2h_bytes_per_step": B * k * (es + 4)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": NCU_TRAFFIC.get((args.workload, B)) if args.impl != "reference" else None,
                     "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": algo_bytes,
                     "step_ms_median": round(statistics.median(step_ms), 5)},
        "clocks": clocks,
    }
    if args.impl == "reference":
        out["impl"] = "reference"
        out["gpu_launches"] = None
        out["cpu_baseline"] = {"value": out["value"], "unit": "Gkeys/s", "cores": 1, "kind": "reference",
                               "sample": "the reference RadiK (topKRadixSelectL, built from its sources for sm_100a) "
                                         "on the GPU; the reference has no CPU implementation of the path"}
        out["e2e"]["h2d_bytes_per_step"] = keys_per_step * es
    else:
        out["impl"] = "radik_b200"
        out["gpu_launches"] = launches_per_step * args.steps
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(x, B, n, k, sorted_, largest, args.cpu_budget)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
