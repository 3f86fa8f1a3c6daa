#!/usr/bin/env python
"""Benchmark of the radix top-k hot path (one JSON line on rank 0).

Headline: plain batched top-k, 256 fp32 rows x 2^20 values, k = 256, largest,
unsorted, values i.i.d. U(0,1) (row r from Philox seed r).  One step is one
radik_topk call over the whole batch.  The inputs (1 GiB) are larger than L2,
so no flush is needed between steps.

The default run (``--workload all``) prints the headline line and, measured
in the same process after the headline's timed region, the rest of the
metric as sub-objects:
  variants  the batched shape at k = 32 / 1024, fp16 keys, sorted output and
            smallest-k ascending (the reference driver's default mode)
  single    one 2^20-key row, k = 256 (U(0,1) seed 0), L2 flushed per launch
  skew      single 2^24-key rows, k = 2^4..2^16, four distributions
  uneven    4096 rows of log-uniform n and k, one radik_topk_rows launch
            replayed from a CUDA graph, beside the plain per-row form
  serving   Poisson arrivals through the continuous-batching server and
            through per-request launches (p50/p99 latency, throughput)
Every part checks its own output after its timed region: values bit-exact
and index sets exact against the CPU oracle (lowest-position ties).  A
mismatch prints the line with "exact": false and exits with status 3.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl radik_b200|reference]
                  [--workload all|batched|batched_k32|batched_k1024|batched_f16|batched_sorted
                              |batched_smallest|single|uneven|skew|serving]

--impl reference runs the reference RadiK (topKRadixSelectL compiled from the
reference's own sources into oracle/_ref/libradik_ref.so) on the same
workloads; the reference has no CPU implementation of the path, and its
uneven figure is its per-row loop (its batch has one K for all rows).
Under torchrun every rank runs the headline on its own GPU (rows are
independent; no collective on the data path): weak scaling.  The
sub-objects are measured at N = 1 only.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gkeys/s & % HBM peak; uneven-batch speedup vs plain per-row; serving p50/p99"

BATCHED = {
    # name: (B, n, k, dtype, sorted, largest, description)
    "batched": (256, 1 << 20, 256, "f32", False, True,
                "plain batched top-k, 256 fp32 rows x 2^20, k=256, largest, unsorted, U(0,1)"),
    "batched_k32": (256, 1 << 20, 32, "f32", False, True,
                    "plain batched top-k, 256 fp32 rows x 2^20, k=32, largest, unsorted, U(0,1)"),
    "batched_k1024": (256, 1 << 20, 1024, "f32", False, True,
                      "plain batched top-k, 256 fp32 rows x 2^20, k=1024, largest, unsorted, U(0,1)"),
    "batched_sorted": (256, 1 << 20, 256, "f32", True, True,
                       "plain batched top-k, 256 fp32 rows x 2^20, k=256, largest, sorted, U(0,1)"),
    "batched_f16": (256, 1 << 20, 256, "f16", False, True,
                    "plain batched top-k, 256 fp16 rows x 2^20, k=256, largest, unsorted, U(0,1) rounded to fp16"),
    "batched_smallest": (256, 1 << 20, 256, "f32", True, False,
                         "plain batched top-k, 256 fp32 rows x 2^20, k=256, smallest, sorted ascending, U(0,1)"),
    "single": (1, 1 << 20, 256, "f32", False, True,
               "plain single-row top-k, one fp32 row of 2^20, k=256, largest, unsorted, U(0,1) seed 0"),
}
VARIANTS = ("batched_k32", "batched_k1024", "batched_f16", "batched_sorted", "batched_smallest")

# DRAM bytes (read + write) per engine launch measured by ncu, keyed by
# workload and rows: (hash of the engine sources captured, bytes, how).  A
# figure whose hash differs from the sources being run describes an older
# kernel and is not reported.
NCU_TRAFFIC = {
    ("batched", 256): ("aa757406f46042f4", 1097415306,
                       "mean of 13 full-size launches"),
    ("batched_f16", 256): ("aa757406f46042f4", 558392202,
                           "mean of 13 full-size launches"),
}


def engine_source_hash() -> str:
    """Hash of the sources that decide what the selection kernel does and moves:
    the engine, its planning kernel and the host code that configures a call
    (not the serving loop, the split-row kernels or the CLI driver)."""
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "radik_b200", "csrc")
    for f in sorted(os.listdir(csrc)):
        if f.endswith((".cu", ".cuh")) and f not in ("radik_cli.cu", "radik_server.cu", "radik_split.cu"):
            with open(os.path.join(csrc, f), "rb") as fh:
                h.update(f.encode() + b"\0" + fh.read())
    return h.hexdigest()[:16]


def traffic_of(workload, rows):
    t = NCU_TRAFFIC.get((workload, rows))
    if t is None:
        return None, "no ncu capture of this workload"
    src, bytes_, how = t
    if src != engine_source_hash():
        return None, f"ncu capture from engine sources {src}; current sources differ"
    return bytes_, f"ncu dram__bytes_read.sum + dram__bytes_write.sum, engine sources {src}, {how}"


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
        return self

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


def _event():
    import torch

    return torch.cuda.Event(enable_timing=True)


def time_steps(step, steps, stream, flush=None):
    """Runs step() `steps` times bracketed by CUDA events on `stream`.
    Returns (whole-span ms, per-step ms list).  With `flush`, the L2 flush
    runs before each step, outside its per-step events but inside the span."""
    import torch

    evs = [(_event(), _event()) for _ in range(steps)]
    t0, t1 = _event(), _event()
    # A device-side delay ahead of the span lets the host enqueue the steps
    # before the GPU reaches them, so the span holds the GPU's time for the
    # K steps and not the host's time to issue the first of them.
    with torch.cuda.stream(stream):
        torch.cuda._sleep(min(200_000 * steps, 100_000_000))
    t0.record(stream)
    for i in range(steps):
        if flush is not None:
            flush()
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize(stream.device)
    return t0.elapsed_time(t1), [a.elapsed_time(b) for a, b in evs]


def roofline(algo_bytes, step_ms, peak, peak_kind, traffic=None, traffic_note=None):
    achieved = algo_bytes / (step_ms / 1e3) / 1e9
    r = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
         "algorithmic_bytes_per_launch": algo_bytes}
    if traffic_note:
        r["traffic_source"] = traffic_note
    return r


# ---------------------------------------------------------------------------
# The two implementations behind one calling convention
# ---------------------------------------------------------------------------
class Ours:
    name = "radik_b200"

    def __init__(self, dev, stream):
        import radik_b200 as rk

        self.rk, self.dev, self.stream = rk, dev, stream

    def dcode(self, dts):
        return {"f32": self.rk.F32, "f16": self.rk.F16}[dts]

    def workspace(self, dts, k, n, B, largest, sorted_):
        import torch

        flags = self.rk.make_flags(largest, sorted_)
        return torch.empty(self.rk.get_radix_select_l_workspace_size(self.dcode(dts), k, n, B, flags),
                           dtype=torch.uint8, device=self.dev)

    def call(self, x, vals, idx, ws, lengths, k, largest, sorted_):
        self.rk.topk_radix_select_l(x, None, vals, idx, ws, lengths, k, largest=largest, ascend=not largest,
                                    need_sorting=sorted_, stream=self.stream)

    def check_status(self, ws):
        self.rk.status(ws, self.stream)


class Ref:
    name = "reference"

    def __init__(self, dev, stream):
        import oracle

        self.ref, self.dev, self.stream = oracle.RefRadik(), dev, stream

    def dcode(self, dts):
        return {"f32": 0, "f16": 1}[dts]

    def workspace(self, dts, k, n, B, largest, sorted_):
        import torch

        return torch.empty(self.ref.workspace_size(self.dcode(dts), k, n, B), dtype=torch.uint8, device=self.dev)

    def call(self, x, vals, idx, ws, lengths, k, largest, sorted_):
        dcode = 1 if x.dtype.itemsize == 2 else 0
        self.ref.topk(dcode, largest, not largest, False, sorted_, x.data_ptr(), vals.data_ptr(), idx.data_ptr(),
                      ws.data_ptr(), lengths, k, self.stream.cuda_stream)

    def check_status(self, ws):
        pass


# ---------------------------------------------------------------------------
# Output checks (run after the timed regions; the oracle is the checker)
# ---------------------------------------------------------------------------
def _canon(vbits, idx, sorted_):
    """Rows of (value bits, indices); unsorted rows ordered by index."""
    if sorted_:
        return vbits, idx
    order = np.argsort(idx, axis=1, kind="stable")
    return np.take_along_axis(vbits, order, 1), np.take_along_axis(idx, order, 1)


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype.itemsize == 4 else a.view(np.uint16)


def check_batched(x_host, B, n, k, sorted_, largest, vals, idx, values_only=False):
    """Compares a uniform batch's device outputs with the oracle."""
    import oracle

    ov, oi = oracle.topk(x_host.reshape(-1), [n] * B, k, flags=oracle.flags_of(largest, sorted_))
    gv = _bits(vals.cpu().numpy()).reshape(B, k)
    gi = idx.cpu().numpy().astype(np.int64).reshape(B, k)
    ov = _bits(ov).reshape(B, k)
    oi = oi.astype(np.int64).reshape(B, k)
    if values_only:
        # the reference breaks ties in arrival order: value multisets only
        bad = int(np.sum(np.any(np.sort(gv, 1) != np.sort(ov, 1), axis=1)))
        return {"rows": B, "exact": bad == 0, "mismatched_rows": bad, "checked": "value multisets vs oracle"}
    gv, gi = _canon(gv, gi, sorted_)
    ov, oi = _canon(ov, oi, sorted_)
    bad = int(np.sum(np.any(gv != ov, axis=1) | np.any(gi != oi, axis=1)))
    return {"rows": B, "exact": bad == 0, "mismatched_rows": bad,
            "checked": "values bit-exact and index sets vs oracle"}


# ---------------------------------------------------------------------------
# Plain batched shapes (headline, variants, single row)
# ---------------------------------------------------------------------------
_INPUT_CACHE = {}


def batched_inputs(B, n, dts):
    """Host rows (numpy) of a batched workload: U(0,1), row r from seed r
    (the single-row workload is row 0: seed 0).  fp16 rows are the
    round-to-nearest of the same draws."""
    from radik_b200 import workloads

    key = (B, n)
    if key not in _INPUT_CACHE:
        _INPUT_CACHE.clear()
        _INPUT_CACHE[key] = workloads.uniform_rows(B, n, 0)
    x = _INPUT_CACHE[key]
    return x.astype(np.float16) if dts == "f16" else x


def run_batched(impl, name, args, dev, stream, world, peak, peak_kind, headline: bool):
    """One batched workload.  Returns (result dict, context for e2e)."""
    import torch

    B, n, k, dts, sorted_, largest, desc = BATCHED[name]
    if args.rows > 0 and name != "single":
        B = args.rows
        desc = desc.replace("256 ", f"{B} ", 1)
    x = batched_inputs(B, n, dts)
    tdtype = torch.float16 if dts == "f16" else torch.float32
    es = 2 if dts == "f16" else 4
    host = torch.from_numpy(x.reshape(-1)).pin_memory() if headline else None
    if host is not None:
        dev_in = host.to(dev)
    else:
        dev_in = torch.from_numpy(x.reshape(-1)).to(dev)
    vals = torch.empty(B * k, dtype=tdtype, device=dev)
    idx = torch.empty(B * k, dtype=torch.int32, device=dev)
    ws = impl.workspace(dts, k, n, B, largest, sorted_)
    lengths = [n] * B

    def step():
        impl.call(dev_in, vals, idx, ws, lengths, k, largest, sorted_)

    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if name == "single" else None
    flush = (lambda: flush_buf.zero_()) if flush_buf is not None else None
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    impl.check_status(ws)
    sampler = ClockSampler(dev.index).start() if headline else None
    if headline:
        time.sleep(0.3)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
    total_ms, step_ms = time_steps(step, args.steps, stream, flush)
    if headline and world > 1:
        torch.distributed.barrier()
    impl.check_status(ws)
    keys = B * n
    algo = keys * es + B * k * (es + 4)
    if flush is not None:
        ms = statistics.median(step_ms)  # per launch; the flushes are outside the per-step events
    else:
        ms = total_ms / args.steps
    res = {"workload": desc, "rows": B, "n": n, "k": k, "dtype": dts, "sorted": sorted_, "largest": largest,
           "ms_per_step": round(ms, 5), "step_ms_median": round(statistics.median(step_ms), 5),
           "gkeys_per_s": round(keys / (ms / 1e3) / 1e9, 3)}
    traffic, tnote = traffic_of(name, B) if impl.name == "radik_b200" else (None, None)
    res["roofline"] = roofline(algo, statistics.mean(step_ms), peak, peak_kind, traffic, tnote)
    ctx = {"B": B, "n": n, "k": k, "dts": dts, "es": es, "sorted": sorted_, "largest": largest, "x": x,
           "host": host, "dev_in": dev_in, "vals": vals, "idx": idx, "step": step, "ws": ws,
           "total_ms": total_ms, "sampler": sampler, "algo": algo, "desc": desc}
    return res, ctx


def parity_batched(impl, ctx):
    return check_batched(ctx["x"], ctx["B"], ctx["n"], ctx["k"], ctx["sorted"], ctx["largest"], ctx["vals"],
                         ctx["idx"], values_only=impl.name == "reference")


# ---------------------------------------------------------------------------
# Skew / adversarial sweep
# ---------------------------------------------------------------------------
def run_skew(impl, args, dev, stream, peak, peak_kind):
    """Single fp32 rows of n = 2^24, k = 2^4..2^16, four distributions
    (U(0,1); 1.0f with random low 8 mantissa bits; Zipf(1.1) ranks; 90% one
    constant + 10% U(0,1)), largest-k, unsorted.  Each case is timed per
    launch with L2 flushed between launches (a 64 MiB row fits L2).  Every
    case's output is checked against the oracle: the top-k of a row for
    every k is a prefix of its sorted top-65536 (ties by lowest position)."""
    import torch

    import oracle
    from radik_b200 import workloads

    n = 1 << 24
    ks = [1 << e for e in range(4, 17)]
    reps = max(3, min(args.steps, 10))
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    vals = torch.empty(max(ks), dtype=torch.float32, device=dev)
    idx = torch.empty(max(ks), dtype=torch.int32, device=dev)
    ws = impl.workspace("f32", max(ks), n, 1, True, False)
    sweep = []
    bad_cases = []
    for dname in workloads.SKEW_DISTRIBUTIONS:
        xh = workloads.skew_row(dname, n, 11)
        x = torch.from_numpy(xh).to(dev)
        ov, oi = oracle.topk(xh, [n], max(ks), flags=oracle.flags_of(True, True))
        ov, oi = _bits(ov), oi.astype(np.int64)
        for k in ks:
            def step():
                impl.call(x, vals, idx, ws, [n], k, True, False)

            def exact():
                gv = _bits(vals[:k].cpu().numpy())
                gi = idx[:k].cpu().numpy().astype(np.int64)
                if impl.name == "reference":
                    return bool(np.array_equal(np.sort(gv), np.sort(ov[:k])))
                o = np.argsort(gi, kind="stable")
                w = np.argsort(oi[:k], kind="stable")
                return bool(np.array_equal(gi[o], oi[:k][w]) and np.array_equal(gv[o], ov[:k][w]))

            for _ in range(args.warmup):
                step()
            _, ts = time_steps(step, reps, stream, lambda: flush_buf.zero_())
            impl.check_status(ws)
            ms = statistics.median(ts)
            if not exact():
                bad_cases.append(f"{dname}/k={k}")
            case = {"dist": dname, "k": k, "ms": round(ms, 4), "gkeys": round(n / (ms / 1e3) / 1e9, 2),
                    "frac": round((n * 4 + k * 8) / (ms / 1e3) / 1e9 / peak, 4)}
            if impl.name == "radik_b200" and not args.no_tune:
                # the autotuner on this case's shape bucket, then the same timing
                choice = impl.rk.autotune(x.view(1, n), k, largest=True, sorted=False, workspace=ws, stream=stream)
                for _ in range(2):
                    step()
                _, ts = time_steps(step, reps, stream, lambda: flush_buf.zero_())
                impl.check_status(ws)
                tms = statistics.median(ts)
                if not exact():
                    bad_cases.append(f"{dname}/k={k} tuned")
                case.update({"tuned_ms": round(tms, 4), "tuned_gkeys": round(n / (tms / 1e3) / 1e9, 2),
                             "tuned": {c: v for c, v in choice.items() if c != "ms"}})
            sweep.append(case)
    if impl.name == "radik_b200" and not args.no_tune:
        impl.rk.autotune_reset()
    g = float(np.exp(np.mean([np.log(c["gkeys"]) for c in sweep])))
    worst = min(sweep, key=lambda c: c["gkeys"])
    fr = float(np.exp(np.mean([np.log(c["frac"]) for c in sweep])))
    tuned = None
    if sweep and "tuned_gkeys" in sweep[0]:
        tg = float(np.exp(np.mean([np.log(c["tuned_gkeys"]) for c in sweep])))
        tuned = {"geomean_gkeys_per_s": round(tg, 2), "speedup_vs_default": round(tg / g, 3),
                 "note": "radik_autotune per case (chunk length, first digit, one-CTA row cap), then re-timed"}
    return {"workload": "skew sweep, single fp32 rows n = 2^24, k = 2^4..2^16, U(0,1) / 1.0f + low-8-bit mantissa "
                        "noise / Zipf(1.1) ranks / 90% constant 0.5 + 10% U(0,1); largest, unsorted",
            "cases": len(sweep), "geomean_gkeys_per_s": round(g, 2), "geomean_frac": round(fr, 4),
            "worst": worst, "tuned": tuned, "l2": "flushed (256 MiB write) before every timed launch", "reps": reps,
            "parity": {"cases": len(sweep), "exact": not bad_cases, "mismatched": bad_cases,
                       "checked": ("value multisets" if impl.name == "reference" else
                                   "values bit-exact and index sets") + " vs oracle"},
            "sweep": sweep}


# ---------------------------------------------------------------------------
# Uneven batch
# ---------------------------------------------------------------------------
def run_uneven(impl, args, dev, stream, peak, peak_kind):
    """4096 fp32 rows, n log-uniform in [2^10, 2^22], k log-uniform in
    [1, min(2048, n)] (lengths and k from seed 7), N(0,1) values generated on
    the device (workloads.uneven_device_values, seed 7).  One step = one
    radik_topk_rows launch over all rows (device descriptors, replayed from a
    CUDA graph).  Beside it the plain per-row form: one call per row, the way
    a RadiK caller handles rows of different k.  For the reference that loop
    is its only form (its batch has one K for all rows)."""
    import ctypes

    import torch

    from radik_b200 import workloads

    B = 4096 if args.rows <= 0 else args.rows
    ns, ks = workloads.uneven_rows(B, 7)
    total_n, n_max, k_max = sum(ns), max(ns), max(ks)
    offs = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    oo = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int64)
    total_out = int(sum(ks))
    dev_in = workloads.uneven_device_values(total_n, 7, dev)
    vals = torch.empty(total_out, dtype=torch.float32, device=dev)
    idx = torch.empty(total_out, dtype=torch.int32, device=dev)
    algo_bytes = total_n * 4 + total_out * 8
    res = {"workload": f"uneven batched top-k, {B} fp32 rows, n log-uniform in [2^10, 2^22], k log-uniform in "
                       f"[1, min(2048, n)], largest, unsorted, N(0,1)",
           "rows": B, "total_keys": total_n, "n_max": n_max, "k_max": k_max,
           "l2": "inputs (%d MiB) larger than L2; no flush" % (total_n * 4 >> 20)}
    if impl.name == "reference":
        ref = impl.ref
        ws = torch.empty(ref.workspace_size(0, k_max, n_max, 1), dtype=torch.uint8, device=dev)
        # The reference reads rows with 16-byte vector loads and takes the
        # alignment of a row from its offset inside the batch, so each row
        # it is given must start 16-byte aligned: rows sit at padded offsets.
        offs_ref = np.zeros(B, np.int64)
        offs_ref[1:] = np.cumsum((np.asarray(ns, np.int64) + 3) // 4 * 4)[:-1]
        padded = torch.zeros(int(offs_ref[-1] + ns[-1] + 4), dtype=torch.float32, device=dev)
        for r in range(B):
            padded[int(offs_ref[r]):int(offs_ref[r]) + ns[r]] = dev_in[int(offs[r]):int(offs[r]) + ns[r]]
        base_v = padded.data_ptr()

        def per_row():
            for r in range(B):
                ref.topk(0, True, False, False, False, base_v + 4 * int(offs_ref[r]), vals.data_ptr() + 4 * int(oo[r]),
                         idx.data_ptr() + 4 * int(oo[r]), ws.data_ptr(), [ns[r]], ks[r], stream.cuda_stream)

        per_row()
        torch.cuda.synchronize(dev)
        span, _ = time_steps(per_row, 2, stream)
        per_row_ms = span / 2
        res.update({"per_row_ms": round(per_row_ms, 3), "gkeys_per_s": round(total_n / (per_row_ms / 1e3) / 1e9, 3),
                    "form": "the reference called once per row (rows re-laid at 16-byte boundaries)"})
        res["roofline"] = roofline(algo_bytes, per_row_ms, peak, peak_kind)
        gv = _bits(vals.cpu().numpy())
        import oracle

        ov, oi = oracle.topk(dev_in.cpu().numpy(), ns, ks, flags=oracle.flags_of(True, False),
                             out_offsets=[int(v) for v in oo])
        ov = _bits(ov)
        bad = sum(1 for r in range(B) if not np.array_equal(np.sort(gv[oo[r]:oo[r] + ks[r]]),
                                                             np.sort(ov[oo[r]:oo[r] + ks[r]])))
        res["parity"] = {"rows": B, "exact": bad == 0, "mismatched_rows": bad, "checked": "value multisets vs oracle"}
        return res
    rk = impl.rk
    L = rk.lib()
    flags = rk.make_flags(True, False)
    desc = np.zeros(B, dtype=[("in_off", "<i8"), ("out_off", "<i8"), ("n", "<i4"), ("k", "<i4")])
    desc["in_off"], desc["out_off"], desc["n"], desc["k"] = offs, oo, ns, ks
    desc_dev = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
    ws = torch.empty(rk.get_rows_workspace_size(rk.F32, B, total_n, n_max, k_max, flags), dtype=torch.uint8,
                     device=dev)

    def call():
        # the current stream: the capture stream while the graph is recorded
        rk._check(L.radik_topk_rows(rk.F32, flags, dev_in.data_ptr(), None, vals.data_ptr(), idx.data_ptr(),
                                    ws.data_ptr(), ws.numel(), desc_dev.data_ptr(), B, total_n, n_max, k_max,
                                    torch.cuda.current_stream(dev).cuda_stream))

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize(dev)
    rk.status(ws, stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        call()
    torch.cuda.synchronize(dev)
    for _ in range(2):
        graph.replay()
    span, step_ms = time_steps(graph.replay, args.steps, stream)
    rk.status(ws, stream)
    ms = span / args.steps
    # parity of the one-launch form
    import oracle

    ov, oi = oracle.topk(dev_in.cpu().numpy(), ns, ks, flags=oracle.flags_of(True, False),
                         out_offsets=[int(v) for v in oo])
    gv, gi = _bits(vals.cpu().numpy()), idx.cpu().numpy().astype(np.int64)
    ov, oi = _bits(ov), oi.astype(np.int64)
    bad = 0
    for r in range(B):
        a, b = int(oo[r]), int(oo[r] + ks[r])
        o = np.argsort(gi[a:b], kind="stable")
        if not (np.array_equal(gi[a:b][o], oi[a:b]) and np.array_equal(gv[a:b][o], ov[a:b])):
            bad += 1
    # the plain per-row form: one radik_topk call per row, arguments prepared up front
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
    span_pr, _ = time_steps(per_row, 2, stream)
    per_row_ms = span_pr / 2
    rk.status(ws_row, stream)
    tuned = None
    if not args.no_tune:
        # the autotuner on the rows form (chunk length, first digit, one-CTA
        # row cap), then a graph captured with the chosen configuration
        choice = rk.autotune_rows(dev_in, desc_dev, B, (total_n, n_max, k_max), total_out, largest=True,
                                  workspace=ws, stream=stream)
        for _ in range(2):
            call()
        torch.cuda.synchronize(dev)
        graph_t = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph_t):
            call()
        torch.cuda.synchronize(dev)
        for _ in range(2):
            graph_t.replay()
        span_t, _ = time_steps(graph_t.replay, args.steps, stream)
        rk.status(ws, stream)
        tms = span_t / args.steps
        gvt, git = _bits(vals.cpu().numpy()), idx.cpu().numpy().astype(np.int64)
        bad_t = 0
        for r in range(B):
            a, b = int(oo[r]), int(oo[r] + ks[r])
            o = np.argsort(git[a:b], kind="stable")
            if not (np.array_equal(git[a:b][o], oi[a:b]) and np.array_equal(gvt[a:b][o], ov[a:b])):
                bad_t += 1
        bad += bad_t
        rk.autotune_reset()
        tuned = {"one_launch_ms": round(tms, 4), "gkeys_per_s": round(total_n / (tms / 1e3) / 1e9, 3),
                 "speedup_vs_default": round(ms / tms, 3), "speedup_vs_per_row": round(per_row_ms / tms, 2),
                 "choice": {c: v for c, v in choice.items() if c != "ms"}, "mismatched_rows": bad_t}
    res.update({"one_launch_ms": round(ms, 4), "gkeys_per_s": round(total_n / (ms / 1e3) / 1e9, 3),
                "per_row_ms": round(per_row_ms, 3),
                "per_row_gkeys_per_s": round(total_n / (per_row_ms / 1e3) / 1e9, 3),
                "speedup_vs_per_row": round(per_row_ms / ms, 2), "cuda_graph": True, "steps": args.steps,
                "launches_per_step": 2, "tuned": tuned})
    res["roofline"] = roofline(algo_bytes, statistics.mean(step_ms), peak, peak_kind)
    res["parity"] = {"rows": B, "exact": bad == 0, "mismatched_rows": bad,
                     "checked": "one-launch form: values bit-exact and index sets vs oracle"}
    return res


# ---------------------------------------------------------------------------
# Serving
# ---------------------------------------------------------------------------
def run_serving(args, dev, stream, peak, peak_kind, requests=10000, rates=(1000, 5000, 10000, 20000, 50000)):
    """Poisson arrivals at 1k..50k requests/s; n in {32000, 128256, 2^20,
    2^24} w.p. {0.4, 0.3, 0.2, 0.1}; k in {1, 50, 1024}; 25% fp16; N(0,1)
    scores already on the device; 40 GiB budget.  The continuous-batching
    server (mode 0) against plain per-request launches (mode 1) on the same
    trace.  Latency = submission to completion seen by the server's worker
    (it polls each batch's event every 2 us).  Every request's result is
    checked against the oracle on its own row."""
    import torch

    import oracle
    import radik_b200 as rk
    from radik_b200 import workloads

    R = requests if args.rows <= 0 else args.rows
    g = workloads.rng(17)
    classes = [32000, 128256, 1 << 20, 1 << 24]
    kset = [1, 50, 1024]
    pools, expect = {}, {}
    for half in (False, True):
        rows_h, lens = [], []
        for ci, n in enumerate(classes):
            bufs = []
            for j in range(4):
                x = workloads.normal(n, 100 * ci + 10 * j + int(half))
                x = x.astype(np.float16) if half else x
                bufs.append(torch.from_numpy(x).to(dev))
                rows_h.append(x)
                lens.append(n)
            pools[(n, half)] = bufs
        flat = np.concatenate(rows_h)
        for k in kset:
            ov, oi = oracle.topk(flat, lens, k, flags=oracle.flags_of(True, False))
            for j, (n, buf) in enumerate([(n, b) for n in classes for b in range(4)]):
                expect[(n, half, buf, k)] = (_bits(ov[j * k:(j + 1) * k]), oi[j * k:(j + 1) * k].astype(np.int64))
    out_f32 = torch.empty(R * 1024, dtype=torch.float32, device=dev)
    out_f16 = torch.empty(R * 1024, dtype=torch.float16, device=dev)
    out_idx = torch.empty(R * 1024, dtype=torch.int32, device=dev)
    ns = g.choice(classes, size=R, p=[0.4, 0.3, 0.2, 0.1])
    ks = g.choice(kset, size=R)
    halves = g.random(R) < 0.25
    keys_total = int(ns.sum())
    flags = rk.make_flags(True, False)
    table = []
    checked, bad = 0, 0

    def verify():
        nonlocal checked, bad
        f32 = _bits(out_f32.cpu().numpy())
        f16 = _bits(out_f16.cpu().numpy())
        ii = out_idx.cpu().numpy().astype(np.int64)
        for i in range(R):
            k = int(ks[i])
            half = bool(halves[i])
            v = (f16 if half else f32)[i * 1024:i * 1024 + k]
            ix = ii[i * 1024:i * 1024 + k]
            ev, ei = expect[(int(ns[i]), half, i % 4, k)]
            o = np.argsort(ix, kind="stable")
            checked += 1
            if not (np.array_equal(ix[o], ei) and np.array_equal(v[o], ev)):
                bad += 1

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
            out_idx.fill_(-2)
            with rk.Server(dev.index, mode=mode, max_n=1 << 24, max_k=1024, budget_bytes=40 << 30) as srv:
                srv.run_trace(items[:16])  # warm-up through the same server
                st0 = srv.stats()
                t0 = time.perf_counter()
                lat = np.asarray(srv.run_trace(items), dtype=np.float64)
                wall = time.perf_counter() - t0
                st1 = srv.stats()
            torch.cuda.synchronize(dev)
            verify()
            span_s = max(float(np.max(arr + lat)) / 1e6, 1e-9)
            row[name] = {"p50_ms": round(float(np.percentile(lat, 50)) / 1e3, 4),
                         "p99_ms": round(float(np.percentile(lat, 99)) / 1e3, 4),
                         "throughput_rps": round(R / span_s, 1),
                         "gkeys_per_s": round(keys_total / span_s / 1e9, 3), "wall_s": round(wall, 3)}
            if mode == 0:
                row[name]["batches"] = st1["batches"] - st0["batches"]
                row[name]["batches_beside_others"] = st1["batches_beside_others"] - st0["batches_beside_others"]
                row[name]["max_batches_in_flight"] = st1["max_batches_in_flight"]
        row["p99_speedup_vs_per_request"] = round(row["per_request"]["p99_ms"] / max(row["batched"]["p99_ms"], 1e-9), 2)
        table.append(row)
    top = table[-1]["batched"]
    sbs = side_by_side(dev)
    return {"workload": "serving: Poisson arrivals at 1k-50k req/s, n in {32000, 128256, 2^20, 2^24} w.p. "
                        "{.4,.3,.2,.1}, k in {1, 50, 1024}, 25% fp16, largest, unsorted, 40 GiB budget",
            "requests_per_rate": R, "latency": "submission to completion seen by the server's worker",
            "p50_ms_at_top_rate": top["p50_ms"], "p99_ms_at_top_rate": top["p99_ms"],
            "gkeys_per_s_at_top_rate": top["gkeys_per_s"],
            "parity": {"requests": checked, "exact": bad == 0, "mismatched": bad,
                       "checked": "every request vs oracle on its own row (values bit-exact, index sets)"},
            "side_by_side": sbs,
            "rates": table}


def side_by_side(dev, reps=20):
    """Two batches of the serving mix on two streams, as the server runs them:
    A = one 2^24-key fp32 request (k = 1024) on three quarters of the SMs,
    B = 16 requests of 32000 keys (k = 50) on the rest
    (radik_topk_rows_ctas; buffers allocated up front, launches through the C
    ABI).  Each rep holds both streams behind a short device-side delay so
    the host has enqueued both calls before the GPU starts them; then each
    call's device span (radik_get_call_span: the GPU global timer when its
    selection kernel's first CTA started and its last CTA ended) shows
    whether the two kernels ran at the same time.  Reported: medians over
    the reps of each call's span alone and side by side, and of the time both
    kernels were running at once.  Both outputs are checked against the
    oracle."""
    import torch

    import oracle
    import radik_b200 as rk
    from radik_b200 import workloads

    L = rk.lib()
    total = rk.engine_ctas(dev.index)
    a_ctas = total * 3 // 4
    b_ctas = total - a_ctas
    flags = rk.make_flags(True, False)
    xa = workloads.normal(1 << 24, 61)
    xb = workloads.normal(16 * 32000, 62)
    calls = {}
    for name, x, rows, ctas in (("a", xa, [(0, 0, 1 << 24, 1024)], a_ctas),
                                ("b", xb, [(j * 32000, j * 50, 32000, 50) for j in range(16)], b_ctas)):
        desc = np.zeros(len(rows), dtype=[("in_off", "<i8"), ("out_off", "<i8"), ("n", "<i4"), ("k", "<i4")])
        for r, (a, o, n, k) in enumerate(rows):
            desc[r] = (a, o, n, k)
        total_n, n_max, k_max = sum(r[2] for r in rows), max(r[2] for r in rows), max(r[3] for r in rows)
        out_n = sum(r[3] for r in rows)
        calls[name] = {
            "x": x, "rows": rows, "ctas": ctas, "bounds": (total_n, n_max, k_max),
            "vals_in": torch.from_numpy(x).to(dev),
            "desc": torch.from_numpy(desc.view(np.uint8).copy()).to(dev),
            "ws": torch.empty(rk.get_rows_workspace_size(rk.F32, len(rows), total_n, n_max, k_max, flags),
                              dtype=torch.uint8, device=dev),
            "vals": torch.empty(out_n, dtype=torch.float32, device=dev),
            "idx": torch.empty(out_n, dtype=torch.int32, device=dev),
            "stream": torch.cuda.Stream(dev)}

    def launch(c):
        total_n, n_max, k_max = c["bounds"]
        rk._check(L.radik_topk_rows_ctas(rk.F32, flags, c["vals_in"].data_ptr(), None, c["vals"].data_ptr(),
                                         c["idx"].data_ptr(), c["ws"].data_ptr(), c["ws"].numel(),
                                         c["desc"].data_ptr(), len(c["rows"]), total_n, n_max, k_max, c["ctas"],
                                         c["stream"].cuda_stream))

    def rep(which):
        for name in which:
            with torch.cuda.stream(calls[name]["stream"]):
                torch.cuda._sleep(200_000)
        for name in which:
            launch(calls[name])
        spans = {name: rk.call_span(calls[name]["ws"], calls[name]["stream"]) for name in which}
        for name in which:
            rk.status(calls[name]["ws"], calls[name]["stream"])
        return spans

    res = {}
    for which in ("a", "b", "ab"):
        for _ in range(3):
            rep(which)
        runs = [rep(which) for _ in range(reps)]
        for name in which:
            key = f"{name}_{'alone' if len(which) == 1 else 'beside'}_us"
            res[key] = round(statistics.median([(r[name][1] - r[name][0]) / 1e3 for r in runs]), 1)
        if which == "ab":
            both = [max(0, min(r["a"][1], r["b"][1]) - max(r["a"][0], r["b"][0])) / 1e3 for r in runs]
            first = [min(r["a"][0], r["b"][0]) for r in runs]
            res["both_running_us"] = round(statistics.median(both), 1)
            res["together_us"] = round(statistics.median([(max(r["a"][1], r["b"][1]) - f) / 1e3
                                                          for r, f in zip(runs, first)]), 1)
            last = runs[-1]
            t0 = min(last["a"][0], last["b"][0])
            res["last_rep_spans_us"] = {n: [round((last[n][0] - t0) / 1e3, 1), round((last[n][1] - t0) / 1e3, 1)]
                                        for n in ("a", "b")}
    res["serial_sum_us"] = round(res["a_alone_us"] + res["b_alone_us"], 1)
    res["overlap_ratio"] = round(res["serial_sum_us"] / max(res["together_us"], 1e-9), 3)
    res["ctas"] = {"a": a_ctas, "b": b_ctas, "device": total}
    bad = 0
    for c in calls.values():
        rows = c["rows"]
        ns, ks, oo = [r[2] for r in rows], [r[3] for r in rows], [r[1] for r in rows]
        ov, oi = oracle.topk(c["x"], ns, ks, flags=oracle.flags_of(True, False), out_offsets=oo)
        gv, gi = _bits(c["vals"].cpu().numpy()), c["idx"].cpu().numpy().astype(np.int64)
        ov = _bits(ov)
        for n, k, o in zip(ns, ks, oo):
            a = np.argsort(gi[o:o + k], kind="stable")
            b = np.argsort(oi[o:o + k], kind="stable")
            if not (np.array_equal(gi[o:o + k][a], oi[o:o + k][b].astype(np.int64))
                    and np.array_equal(gv[o:o + k][a], ov[o:o + k][b])):
                bad += 1
    res["parity"] = {"rows": 17, "exact": bad == 0, "mismatched_rows": bad}
    res["note"] = ("A: one 2^24-key fp32 row, k=1024, on %d CTAs; B: 16 rows of 32000, k=50, on %d CTAs; spans are "
                   "the selection kernels' device spans (GPU global timer); both_running_us = time both kernels "
                   "ran at once; overlap_ratio = (A alone + B alone) / together" % (a_ctas, b_ctas))
    return res


# ---------------------------------------------------------------------------
# CPU baseline (the oracle port on the host cores)
# ---------------------------------------------------------------------------
def cpu_baseline(x: np.ndarray, B, n, k, sorted_, largest, budget_s: float):
    """The oracle (OpenMP nth_element + sort per row) on the host cores."""
    import oracle

    flags = oracle.flags_of(largest, sorted_)
    flat = x.reshape(-1)
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


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="radik_b200", choices=["radik_b200", "reference"])
    ap.add_argument("--workload", default="all", choices=["all"] + sorted(BATCHED) + ["uneven", "skew", "serving"])
    ap.add_argument("--cpu-budget", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the output checks (profiling runs)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuned re-timings (skew, uneven)")
    ap.add_argument("--rows", type=int, default=0, help="override the row count (profiling a smaller case)")
    ap.add_argument("--serving-requests", type=int, default=10000)
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
    stream = torch.cuda.current_stream(dev)
    peak, peak_kind = load_peaks()
    impl = Ref(dev, stream) if args.impl == "reference" else Ours(dev, stream)
    ok = True

    def emit(out):
        if rank == 0:
            print(json.dumps(out), flush=True)

    def base_line(value, unit, ms, dtype, data, config):
        return {"metric": METRIC, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": data, "config": config}

    wl = args.workload
    if wl in ("uneven", "skew", "serving"):
        if world > 1:
            dist.barrier()
        if wl == "serving" and args.impl == "reference":
            emit({"impl": "reference", "unavailable": "the reference has no serving loop; its per-request form "
                                                      "is the mode-1 baseline in this workload's radik_b200 line"})
            return
        sampler = ClockSampler(dev.index).start()
        if wl == "uneven":
            r = run_uneven(impl, args, dev, stream, peak, peak_kind)
            ms = r.get("one_launch_ms", r.get("per_row_ms"))
        elif wl == "skew":
            r = run_skew(impl, args, dev, stream, peak, peak_kind)
            ms = None
        else:
            r = run_serving(args, dev, stream, peak, peak_kind, args.serving_requests)
            ms = r["p50_ms_at_top_rate"]
        clocks = sampler.stop()
        value = r.get("gkeys_per_s", r.get("geomean_gkeys_per_s", r.get("gkeys_per_s_at_top_rate")))
        out = base_line(round(world * value, 3), "Gkeys/s", ms, "f32" if wl != "serving" else "f32/f16",
                        "synthetic, seeded", {"workload": r["workload"]})
        out.update({"e2e": {"value": round(world * value, 3), "unit": "Gkeys/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0, "note": "device-resident inputs"},
                    "roofline": r.get("roofline"), "clocks": clocks, "impl": impl.name,
                    "gpu_launches": None, wl: r})
        ok = r.get("parity", {}).get("exact", True) and r.get("side_by_side", {}).get("parity", {}).get("exact", True)
        emit(out)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        sys.exit(0 if ok else 3)

    # ---- headline (or one batched workload) with e2e, clocks, cpu baseline
    name = "batched" if wl == "all" else wl
    res, ctx = run_batched(impl, name, args, dev, stream, world, peak, peak_kind, headline=True)
    B, n, k, es = ctx["B"], ctx["n"], ctx["k"], ctx["es"]
    host, dev_in, vals, idx, step = ctx["host"], ctx["dev_in"], ctx["vals"], ctx["idx"], ctx["step"]
    vals_h = torch.empty(vals.numel(), dtype=vals.dtype).pin_memory()
    idx_h = torch.empty(idx.numel(), dtype=torch.int32).pin_memory()

    def e2e_step():
        dev_in.copy_(host, non_blocking=True)
        step()
        vals_h.copy_(vals, non_blocking=True)
        idx_h.copy_(idx, non_blocking=True)

    e2e_ms, _ = time_steps(e2e_step, args.steps, stream)
    clocks = ctx["sampler"].stop()
    total_ms = ctx["total_ms"]
    if world > 1:
        t = torch.tensor([total_ms, e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_ms = float(t[0]), float(t[1])
    keys = B * n
    value = world * keys * args.steps / (total_ms / 1e3) / 1e9
    out = base_line(round(value, 3), "Gkeys/s", round(total_ms / args.steps, 5), ctx["dts"],
                    "synthetic: U(0,1) from numpy Philox-4x32-10, row r seed r",
                    {"workload": ctx["desc"], "rows": B, "n": n, "k": k, "sorted": ctx["sorted"],
                     "largest": ctx["largest"], "l2": "inputs (%d MiB) larger than L2; no flush" % (keys * es >> 20)
                     if name != "single" else "L2 flushed (256 MiB write) before every timed launch",
                     "parallelism": f"rows replicated per GPU x{world} (no collective)"})
    if name == "single":
        out["value"] = round(world * res["gkeys_per_s"], 3)
        out["ms_per_step"] = res["ms_per_step"]
    out["e2e"] = {"value": round(world * keys * args.steps / (e2e_ms / 1e3) / 1e9, 3), "unit": "Gkeys/s",
                  "h2d_bytes_per_step": keys * es, "d2h_bytes_per_step": B * k * (es + 4)}
    out["roofline"] = dict(res["roofline"], step_ms_median=res["step_ms_median"])
    out["clocks"] = clocks
    out["impl"] = impl.name
    out["gpu_launches"] = args.steps if impl.name == "radik_b200" else None
    if impl.name == "reference":
        out["cpu_baseline"] = {"value": out["value"], "unit": "Gkeys/s", "cores": 1, "kind": "reference",
                               "sample": "the reference RadiK (topKRadixSelectL, built from its sources for "
                                         "sm_100a) on the GPU; the reference has no CPU implementation of the path"}
    # ---- after the timed regions: output check, CPU baseline, the other parts
    if rank == 0 and world == 1:
        if not args.no_check:
            # the last e2e step left this step's output in vals / idx
            out["parity"] = parity_batched(impl, ctx)
            ok = ok and out["parity"]["exact"]
        if impl.name == "radik_b200" and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(ctx["x"], B, n, k, ctx["sorted"], ctx["largest"], args.cpu_budget)
    if wl == "all" and world == 1:
        del ctx, host, dev_in, vals, idx, vals_h, idx_h
        torch.cuda.empty_cache()
        sampler = ClockSampler(dev.index).start()
        variants = {}
        for v in VARIANTS + ("single",):
            r, c = run_batched(impl, v, args, dev, stream, world, peak, peak_kind, headline=False)
            if not args.no_check:
                r["parity"] = parity_batched(impl, c)
                ok = ok and r["parity"]["exact"]
            del c
            if v == "single":
                out["single"] = r
            else:
                variants[v] = r
        out["variants"] = variants
        _INPUT_CACHE.clear()
        torch.cuda.empty_cache()
        out["skew"] = run_skew(impl, args, dev, stream, peak, peak_kind)
        ok = ok and out["skew"]["parity"]["exact"]
        torch.cuda.empty_cache()
        out["uneven"] = run_uneven(impl, args, dev, stream, peak, peak_kind)
        ok = ok and out["uneven"]["parity"]["exact"]
        torch.cuda.empty_cache()
        if impl.name == "radik_b200":
            out["serving"] = run_serving(args, dev, stream, peak, peak_kind, args.serving_requests)
            ok = ok and out["serving"]["parity"]["exact"] and out["serving"]["side_by_side"]["parity"]["exact"]
        else:
            out["serving"] = {"unavailable": "the reference has no serving loop; its per-request form is the "
                                             "mode-1 baseline in the radik_b200 line"}
        out["clocks_parts"] = sampler.stop()
    emit(out)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    sys.exit(0 if ok else 3)


if __name__ == "__main__":
    main()
