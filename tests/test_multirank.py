"""The N>1 host path of bench.py on CPU: two gloo ranks (127.0.0.1). The step does not shard
(one evolution per device), so --gpus N runs N replicas; what is shared is the max-over-ranks
timing reduction and the rank-0-only reporting, both exercised here without a GPU."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, io, contextlib, datetime
sys.path.insert(0, {root!r})
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
import bench
rank = dist.get_rank()
got = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, device="cpu")
assert got == 15.0, got
# the reference arm reports on rank 0 only; other ranks exit without output or work
buf = io.StringIO()
class A: gpus = 2; steps = 0; warmup = 0
if rank != 0:
    with contextlib.redirect_stdout(buf):
        bench.run_reference_arm(A)
    assert buf.getvalue() == ""
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reduce_max_and_report_on_rank0(tmp_path):
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
