"""The equal-length work-queue layout (UniformB in radik_common.cuh), checked
exhaustively on the host over a grid of row counts, chunk counts, short-chunk
tail rows, FIN flags and FIN delays: every chunk item is decoded exactly once,
every row's FIN exactly once and after the row's last chunk."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_uniform_item_layout(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "item_layout_check")
    subprocess.run([nvcc, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", os.path.join(ROOT, "radik_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "item_layout_check.cu")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad 0" in out.stdout
