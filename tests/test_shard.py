"""Sharding independent evolutions over ranks (hypergraphrewritingengine_b200/shard.py), on the
CPU: the size-balanced assignment, and a batch and a request stream split over two gloo ranks
(127.0.0.1) with a stand-in engine, gathered on rank 0 in input order and equal to the unsplit
run. The GPU engine's own batch path is covered by the -m gpu parity tests."""
import os
import socket
import subprocess
import sys

from hypergraphrewritingengine_b200 import shard
from hypergraphrewritingengine_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_assignment_is_size_balanced_and_deterministic():
    evs = W.config4(n=200)
    sizes = {i: 1 + (i * 7919) % 1000 for i in range(200)}
    est = lambda ev: sizes[int(ev.name.split("-")[1])]  # noqa: E731
    for world in (1, 2, 3, 8):
        owner = shard.assign(evs, world, est)
        assert owner == shard.assign(evs, world, est)
        loads = [0] * world
        for i, r in enumerate(owner):
            loads[r] += sizes[i]
        assert max(loads) - min(loads) <= max(sizes.values())
        idx = [shard.local_share(evs, r, world, est)[0] for r in range(world)]
        assert sorted(i for part in idx for i in part) == list(range(200))


def test_assignment_uses_the_engine_estimate():
    evs = W.config4(n=16)
    owner = shard.assign(evs, 2)     # hgx_estimate_device_bytes through the C-ABI (no device)
    assert set(owner) == {0, 1}


WORKER = r"""
import os, sys, datetime
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
from hypergraphrewritingengine_b200 import shard
from hypergraphrewritingengine_b200 import workloads as W

class FakeResult:
    def __init__(self, ev):
        n = len(ev.roots[0]) * ev.steps
        self.num_states, self.num_events, self.num_classes = n, 2 * n, n
        self.causal, self.branchial, self.truncated = [0] * n, [0] * (n // 2), False
        self.h = np.array([sum(v for e in ev.rules[0][0] for v in e) + 7 * ev.steps, n], dtype=np.uint64)
    def keys(self):
        return {{"state_hashes": self.h, "event_keys": self.h[::-1]}}

class FakeEngine:
    calls = []
    def evolve_batch(self, evs):
        self.calls.append(len(evs))
        return [FakeResult(ev) for ev in evs]

class Rec:
    def __init__(self, t, ev):
        self.arrival, self.admitted, self.finished, self.result = t, t, t + 1, FakeResult(ev)

class FakeServer:
    def run(self, arrivals, realtime=False):
        return [Rec(t, ev) for t, ev in arrivals]

rank = dist.get_rank()
evs = W.config4(n=37)
eng = FakeEngine()
got = shard.evolve_sharded(eng, evs, dist)
mine = sum(FakeEngine.calls)
tot = [None, None] if rank == 0 else None
dist.gather_object(mine, tot, dst=0)
stream = W.config5_stream(23, rate_per_s=100.0, seed=5)
served = shard.serve_sharded(FakeServer, stream, dist, realtime=False)
if rank == 0:
    want = [shard.summary(FakeResult(ev)) for ev in evs]
    assert got == want, "gathered results differ from the unsplit run"
    assert sum(tot) == 37 and min(tot) > 0, tot      # every evolution once, both ranks worked
    assert [s[3] for s in served] == [FakeResult(ev).num_events for _, ev in stream]
    assert [s[0] for s in served] == [t for t, _ in stream]
else:
    assert got is None and served is None
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_batch_and_stream_split_over_two_gloo_ranks(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, o + e
    assert "rank 0 ok" in outs[0][0] and "rank 1 ok" in outs[1][0]
