"""The worker's GPU backend boundary, on the CPU.

* The WXF writer (include/hgx/wxf.hpp) against the Python decoder and, where the reference tree
  is present, the reference's own WXF parser (wxf/wxf.cpp, compiled here from its sources).
* The reference's own build_input (paclet_source/hg_gpu_backend.cpp:25-170), compiled unmodified
  against include/hgx/hg_gpu.hpp: the hg_gpu surface here is a drop-in for the code that fills it.
* include/hgx/gpu_backend.hpp compiles and links against libhgx.so.
The GPU run of the backend itself is tests/test_gpu_backend.py.
"""
import os
import re
import shutil
import subprocess

import pytest

from hypergraphrewritingengine_b200 import wxf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
REF = os.environ.get("HGX_REFERENCE", "/root/reference")
HAVE_REF = os.path.isdir(os.path.join(REF, "wxf")) and os.path.isdir(os.path.join(REF, "paclet_source"))
needs_gxx = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def render(v) -> str:
    """The canonical text form tests/native/wxf_ref_dump.cpp prints."""
    if isinstance(v, bool):
        return str(int(v))
    if isinstance(v, int):
        return str(v)
    if isinstance(v, wxf.Symbol):
        return str(v)
    if isinstance(v, str):
        return '"' + v + '"'
    if isinstance(v, list):
        return "[" + ",".join(render(x) for x in v) + "]"
    if isinstance(v, dict):
        return "<|" + ",".join(render(k) + "->" + render(x) for k, x in v.items()) + "|>"
    raise TypeError(type(v))


def _sample(tmp_path):
    exe = tmp_path / "wxf_writer_sample"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(NATIVE, "wxf_writer_sample.cpp"), "-o", str(exe)])
    out = tmp_path / "sample.wxf"
    subprocess.check_call([str(exe), str(out)])
    return out.read_bytes()


@needs_gxx
def test_wxf_writer_round_trips_through_the_python_decoder(tmp_path):
    v = wxf.loads(_sample(tmp_path))
    assert v["Ints"][-2:] == [2**63 - 1, -2**63]
    assert v["Ints"][:7] == [0, 1, -1, 127, -128, 128, -129]
    assert v["Text"] == "multiway λ step"
    assert v["Nested"] == [[], [1, "two", [3]]]
    assert v["ByState"] == {300: {"IsInitial": 1}, -7: "x"}
    assert v["Flag"] == 0


@needs_gxx
@pytest.mark.skipif(not HAVE_REF, reason="needs the reference tree (its WXF parser)")
def test_wxf_writer_output_parses_with_the_reference_parser(tmp_path):
    data = _sample(tmp_path)
    (tmp_path / "s.wxf").write_bytes(data)
    exe = tmp_path / "wxf_ref_dump"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(REF, "wxf"),
                           "-I", os.path.join(REF, "common", "include"),
                           os.path.join(NATIVE, "wxf_ref_dump.cpp"), os.path.join(REF, "wxf", "wxf.cpp"),
                           "-o", str(exe)])
    out = subprocess.run([str(exe), str(tmp_path / "s.wxf")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == render(wxf.loads(data))


@needs_gxx
@pytest.mark.skipif(not HAVE_REF, reason="needs the reference tree (its build_input)")
def test_reference_build_input_compiles_unmodified_against_the_shim(tmp_path):
    src = open(os.path.join(REF, "paclet_source", "hg_gpu_backend.cpp")).read()
    # the anonymous namespace holding build_input, verbatim
    m = re.search(r"\nnamespace \{\n.*?\n\}  // namespace\n", src, re.S)
    assert m and "hg_gpu::EvolveInput build_input(const GpuJob& job)" in m.group(0)
    tu = tmp_path / "build_input_tu.cpp"
    tu.write_text("#define HG_GPU_BACKEND 1\n"
                  '#include "hgcommon/core.hpp"\n'
                  '#include "graph_marshal.hpp"\n'
                  '#include "hg_gpu_backend.hpp"\n'
                  '#include "hgx/hg_gpu.hpp"\n'
                  "#include <unordered_map>\n#include <stdexcept>\n"
                  + m.group(0) + "\n" + open(os.path.join(NATIVE, "build_input_main.inc")).read()
                  # graph_property_needs lives in the reference's paclet_support.cpp, which needs
                  # its whole CPU engine; the jobs here name no graph property, so it needs none
                  + "\nnamespace HG_NAMESPACE { namespace marshal {\n"
                    "GraphPropertyNeeds graph_property_needs(const std::vector<std::string>& p) {\n"
                    "    if (!p.empty()) throw std::runtime_error(\"no graph properties here\");\n"
                    "    return GraphPropertyNeeds{};\n}\n} }\n")
    from hypergraphrewritingengine_b200 import build
    build.build()
    exe = tmp_path / "build_input_check"
    subprocess.check_call(["g++", "-std=c++17", "-O1",
                           "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(REF, "common", "include"),
                           "-I", os.path.join(REF, "paclet_source"),
                           "-I", os.path.join(REF, "wxf"),
                           str(tu), os.path.join(REF, "wxf", "wxf.cpp"),
                           "-L", os.path.dirname(build.LIB), "-lhgx",
                           "-Wl,-rpath," + os.path.dirname(build.LIB), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.splitlines()
    assert lines[0] == "rules 1 lhs 2 rhs 3 vars 3 3"
    # labels -5, 9, 40 renumbered 0, 1, 2 in order of appearance
    assert lines[1] == "roots 1 edges 3 first 0 1 last 2 0"
    # Full state mode = 2, Full event mode = 1
    assert lines[2] == "steps 4 canon 2 evcanon 1 tr 0 explore 1 edge_identity 1 record 111"
    assert lines[3] == "rejects variable 40: 1"


@needs_gxx
def test_gpu_backend_header_compiles_and_links(tmp_path):
    from hypergraphrewritingengine_b200 import build
    build.build()
    exe = tmp_path / "gpu_backend_test"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                           os.path.join(NATIVE, "gpu_backend_test.cpp"),
                           "-L", os.path.dirname(build.LIB), "-lhgx",
                           "-Wl,-rpath," + os.path.dirname(build.LIB), "-o", str(exe)])
    assert exe.exists()


@needs_gxx
@pytest.mark.skipif(not HAVE_REF, reason="needs the reference tree (its hg_gpu_backend.hpp)")
def test_drop_in_backend_file_compiles_against_the_reference_header(tmp_path):
    """The replacement hg_gpu_backend.cpp shown in INTEGRATION.md, compiled against the
    reference's own hg_gpu_backend.hpp (GpuJob, HostBridge, the run_gpu_evolution declaration)."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```cpp\n(// paclet_source/hg_gpu_backend.cpp\n.*?)```", doc, re.S)
    assert m, "INTEGRATION.md lost the drop-in file"
    src = tmp_path / "hg_gpu_backend.cpp"
    src.write_text(m.group(1))
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-c", "-DHG_GPU_BACKEND=1",
                           "-I", os.path.join(REF, "paclet_source"), "-I", os.path.join(ROOT, "include"),
                           str(src), "-o", str(tmp_path / "hg_gpu_backend.o")])
