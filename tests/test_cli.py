"""The RadiK-compatible driver (radik_b200/bin/test_radik_b200): same argv
and output contract as RadiK's test_radik.out, which its eval scripts parse
with the pattern r"^elapsed: (\\S+) ms$" (eval/libs/radik.py:22-33)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "radik_b200", "bin", "test_radik_b200")


def test_driver_built_and_prints_usage():
    assert os.path.exists(BIN), "run python -m radik_b200.build"
    r = subprocess.run([BIN], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    ["16", "18", "256", "0", "0"],                       # batched, U(0,1)
    ["8", "16", "64", "1", "0", "0", "0"],               # per-task calls, random task lengths
    ["4", "17", "1024", "0", "1", "1"],                  # scaling, U[0.6, 0.7]
    ["4", "16", "32", "0", "0", "2", "1", "1", "0"],     # U[128.6, 128.7], unsorted
    ["2", "16", "100", "0", "0", "3"],                   # Zipf
    ["2", "15", "50", "0", "0", "4"],                    # all zero
])
def test_driver_runs_like_the_reference_binary(args):
    r = subprocess.run([BIN] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == f"batchSize: {args[0]}, K: {args[2]}"
    assert sum(1 for ln in lines if re.match(r"^\[\d+, \d+\]$", ln)) == int(args[0])
    m = [re.match(r"^elapsed: (\S+) ms$", ln.strip()) for ln in lines]
    assert any(m) and float([x for x in m if x][0].group(1)) > 0
