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
    # children hashed through the connectivity shortcut (connected parent, joining RHS)
    assert int(out.stdout.split("(")[1].split()[0]) > 1000, out.stdout
    # children hashed through the uniform-arity initial colours (counts by position)
    assert int(out.stdout.split(", ")[1].split()[0]) > 1000, out.stdout


def _build_compat(tmp_path):
    from hypergraphrewritingengine_b200 import build
    build.build()
    exe = tmp_path / "compat_test"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "native", "compat_test.cpp"),
                           "-L", os.path.dirname(build.LIB), "-lhgx",
                           "-Wl,-rpath," + os.path.dirname(build.LIB), "-o", str(exe)])
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_compat_header_compiles_and_links(tmp_path):
    assert _build_compat(tmp_path).exists()


@pytest.mark.gpu
def test_compat_drop_ins_on_gpu(tmp_path):
    exe = _build_compat(tmp_path)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "compat ok" in out.stdout
