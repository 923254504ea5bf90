"""Host-compiled unit tests of kernel logic shared with the device (CPU only).

The expand kernel's lane-per-child WL hash (csrc/lane_wl.cuh) is a __host__ __device__
function; tests/native/lane_wl_test.cpp compiles it for the host and checks it against the
oracle's WL hash on random parents and matches (AddressSanitizer on).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_lane_wl_matches_oracle(tmp_path):
    exe = tmp_path / "lane_wl_test"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-fsanitize=address", "-I", ROOT,
                           os.path.join(ROOT, "tests", "native", "lane_wl_test.cpp"),
                           os.path.join(ROOT, "oracle", "restate.cpp"), "-o", str(exe)])
    out = subprocess.run([str(exe), "20000"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 / 20000 mismatches" in out.stdout
