"""Per-CTA phase timeline of single radik_topk calls (the timeline build).

Loads libradik_b200_timeline.so (``python -m radik_b200.build --timeline``),
whose engine writes %globaltimer stamps at its phase boundaries into a
device buffer (radik_timeline_attach).  For each shape it

  * times the call back to back from a CUDA graph of 20 calls (``graph_us``:
    GPU time per call with no host gaps),
  * then flushes L2 (a 256 MiB write), runs one call with the stamps on and
    reports, per phase, the minimum / median / maximum over the CTAs that
    stamped it, in microseconds from the earliest CTA start.

  python -m radik_b200.timeline [--shape f32:1:1048576:256 ...] [--json]

A shape is dtype:rows:n:k (largest, unsorted, U(0,1) values).  The phases:

  start          kernel entry
  sample_issue   a whole-CTA sample starts its copies
  sample_in      a whole-CTA sample's keys are in shared memory
  sample_keys    ... and are converted to selection keys
  first_sample   that sample's threshold is published
  item_start     a consumer team starts its last item (its threshold seen)
  chunk_end      a consumer team ends its last pre-filter chunk
  cons_done      the consumer team leaves its item loop
  side_done      the side team leaves its item loop
  fin_start      a finish (FIN) item has seen all of its row's chunks
  fin_begin      the finish has read its row's state
  fin_loaded     candidates are in shared memory
  fin_resolved   the k-th key is found
  fin_emitted    outputs are written
  fin_post       sorting / index mapping / idle fill done
  fin_end        the finish returns
  phase_b        the CTA reaches the grid-wide tail
  end            the CTA leaves the kernel
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

SLOTS = 32
PHASES = {0: "start", 9: "sample_issue", 8: "sample_in", 10: "sample_keys", 1: "first_sample", 14: "item_start",
          15: "chunk_end", 2: "cons_done",
          3: "side_done", 7: "fin_start", 16: "fin_begin", 17: "fin_loaded", 18: "fin_resolved",
          19: "fin_emitted", 20: "fin_post", 4: "fin_end", 5: "phase_b", 6: "end"}
CANDS_SLOT = 31
# per-CTA sums of wait cycles (SM clock) and item counts
WAITS = {21: "prod_side_queue", 22: "prod_cons_queue", 23: "prod_ring", 24: "prod_threshold", 30: "prod_claim",
         25: "cons_stage_data", 26: "cons_threshold", 27: "cons_idle", 28: "fin_wait_chunks", 29: "side_idle"}
COUNTS = {11: "chunk_items", 12: "side_items", 13: "finishes"}
DEFAULT_SHAPES = ("f32:1:1048576:256", "f32:1:16777216:256", "f32:1:16777216:4096", "f32:16:1048576:256",
                  "f32:256:1048576:256", "f16:256:1048576:256", "f32:1:1000:10", "f32:1:100000:256")


def _load_timeline_library():
    import radik_b200 as rk
    from radik_b200 import build

    if rk._lib is not None and rk.LIB_PATH != build.LIB_TIMELINE:
        raise RuntimeError("radik_b200.timeline must load its library before any other radik_b200 call")
    if not os.path.exists(build.LIB_TIMELINE):
        raise ImportError(f"{build.LIB_TIMELINE} is missing; build it with `python -m radik_b200.build --timeline`")
    rk.LIB_PATH = build.LIB_TIMELINE
    return rk, rk.lib()


def measure(shape: str, flush_bytes: int = 256 << 20) -> dict:
    """Graph-timed call time and the per-phase stamps of one flushed call."""
    import numpy as np
    import torch

    rk, L = _load_timeline_library()
    dt, B, n, k = shape.split(":")
    B, n, k = int(B), int(n), int(k)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev).manual_seed(0)
    x = torch.rand(B * n, device=dev, generator=gen)
    if dt == "f16":
        x = x.half()
    elif dt == "bf16":
        x = x.bfloat16()
    code = {"f32": rk.F32, "f16": rk.F16, "bf16": rk.BF16}[dt]
    ws = torch.empty(rk.get_radix_select_l_workspace_size(code, k, n, B, 0), dtype=torch.uint8, device=dev)
    vals = torch.empty(B * k, dtype=x.dtype, device=dev)
    idx = torch.empty(B * k, dtype=torch.int32, device=dev)
    lens = (ctypes.c_int * B)(*([n] * B))
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    stamps = torch.zeros(sm * SLOTS, dtype=torch.int64, device=dev)
    flush = torch.empty(flush_bytes, dtype=torch.uint8, device=dev)

    def call():  # on the current stream, so that a graph capture records it
        rk._check(L.radik_topk(code, rk.LARGEST, x.data_ptr(), None, vals.data_ptr(), idx.data_ptr(),
                               ws.data_ptr(), ws.numel(), lens, B, k, torch.cuda.current_stream(dev).cuda_stream))

    rk._check(L.radik_timeline_attach(None))
    for _ in range(3):
        call()
    torch.cuda.synchronize(dev)
    rk.status(ws)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(20):
            call()
    for _ in range(10):  # keeps the clocks up before the timed replays
        graph.replay()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(10):
        graph.replay()
    b.record(stream)
    torch.cuda.synchronize(dev)
    graph_us = a.elapsed_time(b) * 1e3 / 200
    del graph
    flush.zero_()
    stamps.zero_()
    rk._check(L.radik_timeline_attach(ctypes.c_void_p(stamps.data_ptr())))
    try:
        call()
        torch.cuda.synchronize(dev)
    finally:
        rk._check(L.radik_timeline_attach(None))
    rk.status(ws)
    # nanosecond stamps near 2^60: differences are taken in integers (a
    # float64 of the raw stamp keeps only 256 ns of resolution)
    t = stamps.view(sm, SLOTS).cpu().numpy()
    cands = t[:, CANDS_SLOT].copy()
    ran = t[:, 0] > 0
    t = t[ran]
    t0 = t[:, 0].min()
    phases = {}
    for slot, name in PHASES.items():
        col = t[:, slot]
        col = (col[col > 0] - t0).astype(np.float64) / 1e3
        if col.size:
            phases[name] = [round(float(col.min()), 2), round(float(np.median(col)), 2), round(float(col.max()), 2)]
    mhz = 1965.0  # the B200's maximum SM clock, which an unthrottled run holds
    waits = {}
    for slot, name in WAITS.items():
        col = t[:, slot].astype(np.float64) / mhz
        waits[name] = [round(float(col.min()), 2), round(float(np.median(col)), 2), round(float(col.max()), 2)]
    counts = {name: [int(t[:, slot].min()), float(np.median(t[:, slot])), int(t[:, slot].max())]
              for slot, name in COUNTS.items()}
    return {"shape": {"dtype": dt, "rows": B, "n": n, "k": k}, "ctas": int(ran.sum()),
            "graph_us_per_call": round(graph_us, 2), "finish_candidates_max": int(cands.max()),
            "phases_us_min_median_max": phases, "waits_us_per_cta_min_median_max": waits,
            "counts_per_cta_min_median_max": counts}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--shape", action="append", help="dtype:rows:n:k (repeatable)")
    ap.add_argument("--json", action="store_true", help="one JSON object per shape")
    args = ap.parse_args(argv)
    for shape in args.shape or DEFAULT_SHAPES:
        r = measure(shape)
        if args.json:
            print(json.dumps(r), flush=True)
            continue
        sh = r["shape"]
        print(f"{sh['dtype']} rows={sh['rows']} n={sh['n']} k={sh['k']}: {r['graph_us_per_call']} us per call "
              f"(graph), finish candidates {r['finish_candidates_max']}", flush=True)
        for name, (lo, med, hi) in sorted(r["phases_us_min_median_max"].items(), key=lambda kv: kv[1][1]):
            print(f"    {name:13s} {lo:9.2f} {med:9.2f} {hi:9.2f}")
        print("    waits per CTA (us at the SM clock), min / median / max:")
        for name, (lo, med, hi) in r["waits_us_per_cta_min_median_max"].items():
            print(f"      {name:16s} {lo:9.2f} {med:9.2f} {hi:9.2f}")
        print("    items per CTA:", r["counts_per_cta_min_median_max"])
    return 0


if __name__ == "__main__":
    sys.exit(main())
