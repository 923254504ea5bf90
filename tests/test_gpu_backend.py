"""The worker's GPU backend (include/hgx/gpu_backend.hpp) on the B200: a GpuJob in, the WXF reply
out, decoded and checked against the oracle (C1: the triangle rule at 5 steps, full multiway; C2's
rule at 5 steps under quotient exploration). Counts are the reference's reply fields: NumStates =
classes of the requested state mode (WL classes here), NumEvents, NumCausalEdges = distinct
(producer, consumer) pairs, NumBranchialEdges."""
import os
import subprocess

import numpy as np
import pytest

from hypergraphrewritingengine_b200 import workloads as W
from hypergraphrewritingengine_b200 import wxf
from oracle import pyoracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def backend_exe(tmp_path_factory):
    from hypergraphrewritingengine_b200 import build
    build.build()
    exe = tmp_path_factory.mktemp("backend") / "gpu_backend_test"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "native", "gpu_backend_test.cpp"),
                           "-L", os.path.dirname(build.LIB), "-lhgx",
                           "-Wl,-rpath," + os.path.dirname(build.LIB), "-o", str(exe)])
    return exe


def _reply(exe, job, tmp_path):
    out = tmp_path / f"{job}.wxf"
    r = subprocess.run([str(exe), job, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return wxf.loads(out.read_bytes())


def _pairs(causal):
    return len({(int(p), int(c)) for p, c, _ in causal})


def test_c1_reply_matches_oracle(backend_exe, tmp_path):
    v = _reply(backend_exe, "c1", tmp_path)
    ev = W.config1()
    ref = pyoracle.evolve(ev.rules, ev.roots, 5, quotient=False)
    classes = len(np.unique(ref["state_hash"]))
    assert v["NumStates"] == classes == 20
    assert v["NumEvents"] == len(ref["events"]) == 22203
    assert v["NumBranchialEdges"] == len(ref["branchial"]) == 78045
    assert v["NumCausalEdges"] == _pairs(ref["causal"])
    assert len(v["States"]) == 20 and len(v["Events"]) == 22203
    assert len(v["CausalEdges"]) == v["NumCausalEdges"] and len(v["BranchialEdges"]) == 78045
    # every event's canonical endpoints are listed states; one initial state at step 0
    for e in v["Events"].values():
        assert e["CanonicalInputState"] in v["States"] and e["CanonicalOutputState"] in v["States"]
        assert len(e) == 9 and len(e["ConsumedEdges"]) == 2 and len(e["ProducedEdges"]) == 3
    init = [s for s in v["States"].values() if s["IsInitial"]]
    assert len(init) == 1 and init[0]["Step"] == 0 and len(init[0]["Edges"]) == 3
    # the class representatives' edge counts follow their step (3 edges + 1 per event)
    for s in v["States"].values():
        assert len(s["Edges"]) == 3 + s["Step"]


def test_c1_genesis_reply(backend_exe, tmp_path):
    v = _reply(backend_exe, "c1-genesis", tmp_path)
    plain = _reply(backend_exe, "c1", tmp_path)
    assert len(v["Events"]) == 22203 + 1
    genesis = [e for e in v["Events"].values() if e["RuleIndex"] == -1]
    assert len(genesis) == 1 and len(genesis[0]["ProducedEdges"]) == 3
    gid = genesis[0]["Id"]
    # the genesis event causes every event that consumes an initial edge
    initial = set(genesis[0]["ProducedEdges"])
    consumers = {e["Id"] for e in v["Events"].values() if set(e["ConsumedEdges"]) & initial}
    added = {c["To"] for c in v["CausalEdges"] if c["From"] == gid}
    assert added == consumers and v["NumCausalEdges"] == plain["NumCausalEdges"] + len(consumers)
    assert len(v["StateBitvectors"]) == 22204
    # every edge of every recorded state is in GlobalEdges with its vertices
    ge = {row[0]: row[1:] for row in v["GlobalEdges"]}
    for ids in list(v["StateBitvectors"].values())[::997]:
        assert all(i in ge and len(ge[i]) == 2 for i in ids)


def test_c2_quotient_reply_matches_oracle(backend_exe, tmp_path):
    v = _reply(backend_exe, "c2q", tmp_path)
    ev = W.config2(5)
    ref = pyoracle.evolve(ev.rules, ev.roots, 5, quotient=True)
    assert v["NumStates"] == ref["classes"]
    assert v["NumEvents"] == len(ref["events"])
    assert v["NumBranchialEdges"] == len(ref["branchial"])
    assert v["NumCausalEdges"] == _pairs(ref["causal"])
    hashes = sorted(s["CanonicalHash"] & (2**64 - 1) for s in v["States"].values())
    assert hashes == sorted(int(h) for h in np.unique(ref["state_hash"]))
    assert all(len(e) == 7 for e in v["Events"].values())   # EventsMinimal
