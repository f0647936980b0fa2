"""CTA range splits of the streamed CG (host code, csrc/stream_partition.h):
valid and deterministic ranges, the two-phase objective no worse than equal
summed weights, and the per-range bound kept (tests/stream_partition_test.cpp,
compiled here with the host compiler)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_stream_partition_properties(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "stream_partition_test")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "higher_order_embedded_fem_b200", "csrc"),
                           os.path.join(ROOT, "tests", "stream_partition_test.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
