"""Build recipe for the in-tree CUDA library (sm_100a) and the test checkers.

``build()`` compiles radik_b200/libradik_b200.so with nvcc for sm_100a and, via
oracle/Makefile, the CPU oracle (and the reference RadiK wrapper when the
reference sources are present).  The .so files stay in the tree so they ship
with it; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libradik_b200.so")
# The timeline build: the same sources with RADIK_TIMELINE, whose engine
# writes per-CTA phase stamps (radik_timeline_attach, radik_b200/timeline.py).
LIB_TIMELINE = os.path.join(HERE, "libradik_b200_timeline.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in (
    "radik_engine_f32.cu", "radik_engine_f16.cu", "radik_engine_bf16.cu", "radik_plan.cu", "radik_api.cu",
    "radik_server.cu", "radik_split.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("radik_common.cuh", "radik_engine.cuh")] + [
    os.path.join(ROOT, "include", "radik_b200.h")]
OBJ_DIR = os.path.join(ROOT, "_build")

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build radik_b200")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False, timeline: bool = False) -> str:
    """Compiles each translation unit in parallel, then links the .so
    (timeline=True: the timeline build, libradik_b200_timeline.so)."""
    lib = LIB_TIMELINE if timeline else LIB
    obj_dir = os.path.join(OBJ_DIR, "timeline") if timeline else OBJ_DIR
    if not (force or _stale(lib, SOURCES + HEADERS)):
        return lib
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(obj_dir, exist_ok=True)
    nvcc = _nvcc()
    inc = "-I" + os.path.join(ROOT, "include")
    extra = ["-DRADIK_TIMELINE"] if timeline else []

    def compile_one(src: str) -> str:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        if not force and not _stale(obj, [src] + HEADERS + [__file__]):
            return obj  # up to date: the engine units take minutes each
        cmd = [nvcc, *NVCC_FLAGS, *extra, inc, "-c", "-o", obj, src]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib + ".tmp", *objs],
                   check=True)
    os.replace(lib + ".tmp", lib)
    return lib


CLI_SRC = os.path.join(HERE, "csrc", "radik_cli.cu")
CLI_BIN = os.path.join(HERE, "bin", "test_radik_b200")


def build_cli(force: bool = False, verbose: bool = False) -> str:
    """The RadiK-compatible benchmark driver (links libradik_b200.so)."""
    deps = [CLI_SRC, LIB, os.path.join(ROOT, "include", "topk_radixselect.h")]
    if not (force or _stale(CLI_BIN, deps)):
        return CLI_BIN
    os.makedirs(os.path.dirname(CLI_BIN), exist_ok=True)
    cmd = [_nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ROOT, "include"),
           "-o", CLI_BIN + ".tmp", CLI_SRC, "-L" + HERE, "-lradik_b200", "-lcurand", "-Xlinker", "-rpath",
           "-Xlinker", "$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(CLI_BIN + ".tmp", CLI_BIN)
    return CLI_BIN


# Where the build container keeps the reference checkout's radik/ directory
# (read-only; only the test checker oracle/_ref is built from it).  The GPU
# runs use the prebuilt oracle/_ref and never read it.
REFERENCE_SOURCES = os.path.join(os.sep, "root", "reference", "radik")


def build_oracle(verbose: bool = False) -> None:
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("make not found")
    out = None if verbose else subprocess.DEVNULL
    cmd = [make, "-s", "-C", os.path.join(ROOT, "oracle"), "all"]
    ref = os.environ.get("RADIK_REF") or (REFERENCE_SOURCES if os.path.isdir(REFERENCE_SOURCES) else "")
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, stdout=out)


def build(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_library(force=force, verbose=verbose, timeline=True)
    build_cli(force=force, verbose=verbose)
    build_oracle(verbose=verbose)


if __name__ == "__main__":
    if "--timeline" in sys.argv:
        build_library(force="--force" in sys.argv, verbose=True, timeline=True)
    else:
        build(force="--force" in sys.argv, verbose=True)
