#!/usr/bin/env python
"""Benchmark of the radix top-k hot path (one JSON line on rank 0).

Default workload: plain batched top-k, 256 fp32 rows x 2^20 values, k = 256,
largest, unsorted, values i.i.d. U(0,1) (row r from Philox seed r).  One step
is one radik_topk call over the whole batch.  The inputs (1 GiB) are larger
than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl radik_b200|reference]
                  [--workload batched|batched_k32|batched_k1024|batched_f16|batched_sorted|single
                              |uneven|skew|serving]

uneven: 4096 rows of log-uniform n and per-row k, one radik_topk_rows launch
replayed from a CUDA graph, beside the plain per-row form.  skew: single
2^24 rows, k = 2^4..2^16, four distributions.  serving: Poisson arrivals
through the continuous-batching server and through per-request launches.

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
    ("batched", 256): 4 * (270063360 + 4457728),  # profiles/engine_kernel_f32_64x1M_k256_full.md
    ("batched", 64): 270063360 + 4457728,
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


def _events(n):
    import torch

    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def run_uneven(args, dev, world, rank):
    """Uneven batched top-k: 4096 fp32 rows, n log-uniform in [2^10, 2^22], k
    log-uniform in [1, min(2048, n)], N(0,1) values.  One step = one
    radik_topk_rows launch over all rows (device descriptors, replayed from a
    CUDA graph).  Reported beside it: the plain per-row form (one radik_topk
    call per row, the way a RadiK caller handles rows of different k)."""
    import ctypes

    import torch

    from radik_b200 import workloads

    B = 4096 if args.rows <= 0 else args.rows
    ns, ks = workloads.uneven_rows(B, 7)
    total_n, n_max, k_max = sum(ns), max(ns), max(ks)
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int64)
    total_out = int(sum(ks))
    x = np.empty(total_n, np.float32)
    for r in range(B):
        x[offs[r]:offs[r] + ns[r]] = workloads.normal(ns[r], 1000 + r)
    host = torch.from_numpy(x).pin_memory()
    dev_in = host.to(dev)
    stream = torch.cuda.current_stream(dev)
    desc = np.zeros(B, dtype=[("in_off", "<i8"), ("out_off", "<i8"), ("n", "<i4"), ("k", "<i4")])
    desc["in_off"], desc["out_off"], desc["n"], desc["k"] = offs, oo, ns, ks
    desc_dev = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
    algo_bytes = total_n * 4 + total_out * 8
    peak, peak_kind = load_peaks()
    out = {"metric": "Gkeys/s & % HBM peak; uneven-batch speedup vs plain per-row; serving p50/p99",
           "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: N(0,1) from numpy Philox-4x32-10, row r seed 1000 + r; lengths/k seed 7",
           "config": {"workload": f"uneven batched top-k, {B} fp32 rows, n log-uniform in [2^10, 2^22], "
                                  f"k log-uniform in [1, min(2048, n)], largest, unsorted",
                      "rows": B, "total_keys": total_n, "n_max": n_max, "k_max": k_max,
                      "l2": "inputs (%d MiB) larger than L2; no flush" % (total_n * 4 >> 20),
                      "parallelism": f"rows replicated per GPU x{world} (no collective)"}}
    vals = torch.empty(total_out, dtype=torch.float32, device=dev)
    idx = torch.empty(total_out, dtype=torch.int32, device=dev)

    if args.impl == "reference":
        import oracle

        ref = oracle.RefRadik()
        ws = torch.empty(ref.workspace_size(0, k_max, n_max, 1), dtype=torch.uint8, device=dev)

        # The reference reads rows with 16-byte vector loads and takes the
        # alignment of a row from its offset inside the batch, so a row pointer
        # of its own must be 16-byte aligned: its rows sit at padded offsets.
        offs_ref = np.zeros(B, np.int64)
        offs_ref[1:] = np.cumsum((np.asarray(ns, np.int64) + 3) // 4 * 4)[:-1]
        padded = torch.zeros(int(offs_ref[-1] + ns[-1] + 4), dtype=torch.float32, device=dev)
        for r in range(B):
            padded[int(offs_ref[r]):int(offs_ref[r]) + ns[r]] = dev_in[int(offs[r]):int(offs[r]) + ns[r]]

        def step(inp):
            base_v = padded.data_ptr()
            for r in range(B):
                ref.topk(0, True, False, False, False, base_v + 4 * int(offs_ref[r]), vals.data_ptr() + 4 * int(oo[r]),
                         idx.data_ptr() + 4 * int(oo[r]), ws.data_ptr(), [ns[r]], ks[r], stream.cuda_stream)
        launches = None
    else:
        import radik_b200 as rk

        L = rk.lib()
        flags = rk.make_flags(True, False)
        ws = torch.empty(rk.get_rows_workspace_size(rk.F32, B, total_n, n_max, k_max, flags), dtype=torch.uint8,
                         device=dev)

        def call(inp):
            rk._check(L.radik_topk_rows(rk.F32, flags, inp.data_ptr(), None, vals.data_ptr(), idx.data_ptr(),
                                        ws.data_ptr(), ws.numel(), desc_dev.data_ptr(), B, total_n, n_max, k_max,
                                        torch.cuda.current_stream(dev).cuda_stream))

        for _ in range(args.warmup):
            call(dev_in)
        torch.cuda.synchronize(dev)
        rk.status(ws, stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            call(dev_in)
        torch.cuda.synchronize(dev)

        def step(inp):
            graph.replay()
        launches = 2  # planning kernel + selection engine (the workspace clear is a memset node)
        # plain per-row form: one radik_topk call per row, arguments prepared up front
        ws_row = torch.empty(rk.get_radix_select_l_workspace_size(rk.F32, k_max, n_max, 1, flags), dtype=torch.uint8,
                             device=dev)
        lens = [(ctypes.c_int * 1)(n) for n in ns]
        v0, o0, i0, w0 = dev_in.data_ptr(), vals.data_ptr(), idx.data_ptr(), ws_row.data_ptr()
        wsz, sh = ws_row.numel(), stream.cuda_stream

        def per_row():
            for r in range(B):
                L.radik_topk(rk.F32, flags, v0 + 4 * int(offs[r]), None, o0 + 4 * int(oo[r]), i0 + 4 * int(oo[r]),
                             w0, wsz, lens[r], 1, ks[r], sh)
        per_row()
        torch.cuda.synchronize(dev)
        ev = _events(1)[0]
        ev[0].record(stream)
        per_row()
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        per_row_ms = ev[0].elapsed_time(ev[1])
        rk.status(ws_row, stream)

    for _ in range(args.warmup):
        step(dev_in)
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(dev.index)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    evs = _events(args.steps)
    t0, t1 = _events(1)[0]
    t0.record(stream)
    for i in range(args.steps):
        evs[i][0].record(stream)
        step(dev_in)
        evs[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    total_ms = t0.elapsed_time(t1)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    vals_h = torch.empty(total_out, dtype=torch.float32).pin_memory()
    idx_h = torch.empty(total_out, dtype=torch.int32).pin_memory()
    e0, e1 = _events(1)[0]
    e_steps = max(1, min(args.steps, 5))
    e0.record(stream)
    for i in range(e_steps):
        dev_in.copy_(host, non_blocking=True)
        step(dev_in)
        vals_h.copy_(vals, non_blocking=True)
        idx_h.copy_(idx, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / e_steps
    clocks = sampler.stop()
    if world > 1:
        t = torch.tensor([total_ms, e2e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms, e2e_ms = float(t[0]), float(t[1])
    ms = total_ms / args.steps
    out["value"] = round(world * total_n / (ms / 1e3) / 1e9, 3)
    out["ms_per_step"] = round(ms, 5)
    out["e2e"] = {"value": round(world * total_n / (e2e_ms / 1e3) / 1e9, 3), "unit": "Gkeys/s",
                  "h2d_bytes_per_step": total_n * 4, "d2h_bytes_per_step": total_out * 8}
    achieved = algo_bytes / (statistics.mean(step_ms) / 1e3) / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(achieved / peak, 4), "traffic": None, "peak_source": f"{peak_kind} hbm_gbs",
                       "algorithmic_bytes_per_launch": algo_bytes}
    out["clocks"] = clocks
    if args.impl == "reference":
        out["impl"] = "reference"
        out["gpu_launches"] = None
        out["cpu_baseline"] = {"value": out["value"], "unit": "Gkeys/s", "cores": 1, "kind": "reference",
                               "sample": "the reference RadiK called once per row (its batched API has one K for "
                                         "all rows), built from its sources for sm_100a, on the GPU"}
    else:
        out["impl"] = "radik_b200"
        out["gpu_launches"] = launches * args.steps
        out["uneven"] = {"one_launch_ms": round(ms, 4), "per_row_ms": round(per_row_ms, 3),
                         "per_row_gkeys": round(total_n / (per_row_ms / 1e3) / 1e9, 3),
                         "speedup_vs_per_row": round(per_row_ms / ms, 2), "cuda_graph": True}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            import oracle

            rows = min(B, 256)
            t = time.perf_counter()
            oracle.topk(x[:int(offs[rows - 1] + ns[rows - 1])], ns[:rows], ks[:rows], flags=oracle.flags_of(True, False),
                        out_offsets=[int(v) for v in oo[:rows]])
            dt = time.perf_counter() - t
            keys = int(sum(ns[:rows]))
            out["cpu_baseline"] = {"value": round(keys / dt / 1e9, 4), "unit": "Gkeys/s", "cores": oracle.max_threads(),
                                   "kind": "port", "sample": f"the first {rows} rows ({keys} keys), OpenMP "
                                                             f"nth_element per row"}
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_skew(args, dev, world, rank):
    """Skew / adversarial sweep: single fp32 rows of n = 2^24, k = 2^4 .. 2^16,
    four distributions (U(0,1); 1.0f with random low 8 mantissa bits; Zipf(1.1)
    ranks; 90% one constant + 10% U(0,1)), largest-k, unsorted.  Each case is
    timed per launch with L2 flushed between launches (a 64 MiB row fits L2).
    value = geometric mean Gkeys/s over the cases; the table is in "sweep"."""
    import torch

    from radik_b200 import workloads

    n = 1 << 24
    ks = [1 << e for e in range(4, 17)]
    dists = ["uniform", "mantissa_noise", "zipf", "constant_heavy"]
    reps = max(3, min(args.steps, 10))
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    vals = torch.empty(max(ks), dtype=torch.float32, device=dev)
    idx = torch.empty(max(ks), dtype=torch.int32, device=dev)
    if args.impl == "reference":
        import oracle

        ref = oracle.RefRadik()
        ws = torch.empty(ref.workspace_size(0, max(ks), n, 1), dtype=torch.uint8, device=dev)

        def call(x, k):
            ref.topk(0, True, False, False, False, x.data_ptr(), vals.data_ptr(), idx.data_ptr(), ws.data_ptr(), [n], k,
                     stream.cuda_stream)
    else:
        import radik_b200 as rk

        flags = rk.make_flags(True, False)
        ws = torch.empty(rk.get_radix_select_l_workspace_size(rk.F32, max(ks), n, 1, flags), dtype=torch.uint8,
                         device=dev)

        def call(x, k):
            rk.topk_radix_select_l(x, None, vals, idx, ws, [n], k, largest=True, ascend=False, need_sorting=False,
                                   stream=stream)
    sweep = []
    clocks = None
    sampler = ClockSampler(dev.index)
    sampler.start()
    for dname in dists:
        x = torch.from_numpy(workloads.skew_row(dname, n, 11)).to(dev)
        for k in ks:
            for _ in range(args.warmup):
                call(x, k)
            ts = []
            for _ in range(reps):
                flush.zero_()
                a, b = _events(1)[0]
                a.record(stream)
                call(x, k)
                b.record(stream)
                torch.cuda.synchronize(dev)
                ts.append(a.elapsed_time(b))
            ms = statistics.median(ts)
            sweep.append({"dist": dname, "k": k, "ms": round(ms, 4), "gkeys": round(n / (ms / 1e3) / 1e9, 2)})
        if args.impl != "reference":
            rk.status(ws, stream)
    clocks = sampler.stop()
    g = float(np.exp(np.mean([np.log(c["gkeys"]) for c in sweep])))
    total_ms = sum(c["ms"] for c in sweep)
    peak, peak_kind = load_peaks()
    ach = float(np.exp(np.mean([np.log((n * 4 + c["k"] * 8) / (c["ms"] / 1e3) / 1e9) for c in sweep])))
    out = {"metric": "Gkeys/s & % HBM peak; uneven-batch speedup vs plain per-row; serving p50/p99",
           "value": round(world * g, 3), "unit": "Gkeys/s", "n_gpus": world, "steps": reps, "warmup": args.warmup,
           "ms_per_step": round(total_ms / len(sweep), 5), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: four distributions from numpy Philox-4x32-10, seed 11",
           "config": {"workload": "skew sweep, single fp32 rows n = 2^24, k = 2^4..2^16, U(0,1) / 1.0f + low-8-bit "
                                  "mantissa noise / Zipf(1.1) ranks / 90% constant 0.5 + 10% U(0,1); largest, "
                                  "unsorted; value = geometric mean over the 52 cases",
                      "n": n, "l2": "L2 flushed (256 MiB write) before every timed launch",
                      "parallelism": f"replicated per GPU x{world}"},
           "e2e": {"value": round(world * g, 3), "unit": "Gkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                   "note": "device-resident inputs; the end-to-end copy cost is the batched workload's"},
           "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(ach / peak, 4), "traffic": None, "peak_source": f"{peak_kind} hbm_gbs",
                        "algorithmic_bytes_per_launch": "n*4 + k*8"},
           "clocks": clocks, "sweep": sweep}
    out["impl"] = "reference" if args.impl == "reference" else "radik_b200"
    out["gpu_launches"] = None if args.impl == "reference" else len(sweep) * (args.warmup + reps)
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_serving(args, dev, world, rank):
    """Serving loop: Poisson arrivals at 1k..50k requests/s; n in {32000,
    128256, 2^20, 2^24} w.p. {0.4, 0.3, 0.2, 0.1}; k in {1, 50, 1024}; 25% fp16;
    N(0,1) scores already on the device; 40 GiB budget.  The continuous-
    batching server (radik_server, mode 0) against plain per-request launches
    (mode 1) on the same trace.  Latency = submission to completion."""
    import torch

    import radik_b200 as rk
    from radik_b200 import workloads

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop; its per-request "
                              "form is the mode-1 baseline reported in this workload's radik_b200 line"}))
        return
    rates = [1000, 5000, 10000, 20000, 50000]
    R = 10000 if args.rows <= 0 else args.rows
    g = workloads.rng(17)
    classes = [32000, 128256, 1 << 20, 1 << 24]
    pools = {}
    for ci, n in enumerate(classes):
        for half in (False, True):
            bufs = []
            for j in range(4):
                x = workloads.normal(n, 100 * ci + 10 * j + int(half))
                bufs.append(torch.from_numpy(x.astype(np.float16) if half else x).to(dev))
            pools[(n, half)] = bufs
    out_f32 = torch.empty(R * 1024, dtype=torch.float32, device=dev)
    out_f16 = torch.empty(R * 1024, dtype=torch.float16, device=dev)
    out_idx = torch.empty(R * 1024, dtype=torch.int32, device=dev)
    ns = g.choice(classes, size=R, p=[0.4, 0.3, 0.2, 0.1])
    ks = g.choice([1, 50, 1024], size=R)
    halves = g.random(R) < 0.25
    keys_total = int(ns.sum())
    flags = rk.make_flags(True, False)
    table = []
    sampler = ClockSampler(dev.index)
    sampler.start()
    for rate in rates:
        gaps = g.exponential(1e6 / rate, size=R)
        arr = np.cumsum(gaps) - gaps[0]
        items = []
        for i in range(R):
            n, k, half = int(ns[i]), int(ks[i]), bool(halves[i])
            x = pools[(n, half)][i % 4]
            vo = (out_f16 if half else out_f32)[i * 1024:]
            items.append(rk.TraceItem(float(arr[i]), rk.F16 if half else rk.F32, flags, x.data_ptr(), n, k,
                                      vo.data_ptr(), out_idx[i * 1024:].data_ptr()))
        row = {"rate_rps": rate, "requests": R}
        for mode, name in ((0, "batched"), (1, "per_request")):
            with rk.Server(dev.index, mode=mode, max_n=1 << 24, max_k=1024, budget_bytes=40 << 30) as srv:
                # warm-up: a few requests through the same server
                srv.run_trace(items[:16])
                t0 = time.perf_counter()
                lat = np.asarray(srv.run_trace(items), dtype=np.float64)
                wall = time.perf_counter() - t0
            span_s = max(float(np.max(arr + lat)) / 1e6, 1e-9)
            row[name] = {"p50_ms": round(float(np.percentile(lat, 50)) / 1e3, 4),
                         "p99_ms": round(float(np.percentile(lat, 99)) / 1e3, 4),
                         "throughput_rps": round(R / span_s, 1),
                         "gkeys_per_s": round(keys_total / span_s / 1e9, 3), "wall_s": round(wall, 3)}
        row["p99_speedup_vs_per_request"] = round(row["per_request"]["p99_ms"] / max(row["batched"]["p99_ms"], 1e-9), 2)
        table.append(row)
    clocks = sampler.stop()
    top = table[-1]["batched"]
    peak, peak_kind = load_peaks()
    out = {"metric": "Gkeys/s & % HBM peak; uneven-batch speedup vs plain per-row; serving p50/p99",
           "value": top["gkeys_per_s"], "unit": "Gkeys/s", "n_gpus": world, "steps": R, "warmup": 16,
           "ms_per_step": top["p50_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32/f16", "data": "synthetic: N(0,1) score pools (numpy Philox), Poisson arrivals seed 17",
           "config": {"workload": "serving: Poisson arrivals at 1k-50k req/s, n in {32000, 128256, 2^20, 2^24} "
                                  "w.p. {.4,.3,.2,.1}, k in {1, 50, 1024}, 25% fp16, largest, unsorted, 40 GiB budget; "
                                  "value = keys served per second at 50k req/s",
                      "requests_per_rate": R, "l2": "score pools larger than L2 (64 MiB rows)",
                      "parallelism": "one server per GPU"},
           "e2e": {"value": top["gkeys_per_s"], "unit": "Gkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                   "note": "requests' scores are produced on the device; latency is submission to completion"},
           "roofline": {"bound": "hbm", "achieved": round(top["gkeys_per_s"] * 1e9 * 3.5 / 1e9, 1), "peak": peak,
                        "unit": "GB/s", "frac": round(top["gkeys_per_s"] * 3.5 / peak, 4), "traffic": None,
                        "peak_source": f"{peak_kind} hbm_gbs", "note": "offered load, not a bound: mean 3.5 B/key"},
           "clocks": clocks, "serving": table, "impl": "radik_b200", "gpu_launches": None}
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="radik_b200", choices=["radik_b200", "reference"])
    ap.add_argument("--workload", default="batched", choices=sorted(WORKLOADS) + ["uneven", "skew", "serving"])
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
    if args.workload == "uneven":
        run_uneven(args, dev, world, rank)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload in ("skew", "serving"):
        (run_skew if args.workload == "skew" else run_serving)(args, dev, world, rank)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

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
