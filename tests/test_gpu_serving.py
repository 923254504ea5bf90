"""Continuous batching: every request's result is the same served in the mix as evolved alone
(and as the oracle's), whatever the admission pattern. Exact comparison (integer work)."""
import pytest

from hypergraphrewritingengine_b200 import workloads as W
from hypergraphrewritingengine_b200.serve import Server, serve_plain, summarize
from oracle import pyoracle
from parity import assert_same, norm_gpu, norm_oracle

pytestmark = pytest.mark.gpu


def _stream(n, seed):
    s = W.config5_stream(n, rate_per_s=1000.0, seed=seed, max_states=512)
    # a zero-step request and a request that reuses an earlier one's input
    s.append((s[-1][0] + 1e-3, W.Evolution(rules=s[0][1].rules, roots=s[0][1].roots, steps=0,
                                           max_states=512)))
    s.append((s[-1][0] + 1e-3, s[3][1]))
    return s


@pytest.mark.parametrize("admit_per_step", [1, 4, 64])
def test_served_results_equal_alone(engine, admit_per_step):
    stream = _stream(40, seed=7 + admit_per_step)
    recs = Server(engine).run(stream, realtime=False, admit_per_step=admit_per_step)
    assert all(r.finished >= r.admitted >= 0 for r in recs)
    for rec, (_, ev) in zip(recs, stream):
        alone = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        a, b = norm_gpu(rec.result), norm_gpu(alone)
        assert_same(a, b, f"request {rec.rid}")
        assert rec.result.truncated == alone.truncated
        if rec.rid % 5 == 0:
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(a, norm_oracle(ref), f"request {rec.rid} vs oracle")


def test_served_state_records_match(engine):
    stream = _stream(12, seed=3)
    recs = Server(engine).run(stream, realtime=False, admit_per_step=2)
    for rec in recs:
        res = rec.result
        for s in range(0, res.num_states, 11):
            assert pyoracle.wl_hash(res.state_edges(s)) == int(res.state_hash[s])


def test_realtime_serving_and_plain_agree(engine):
    stream = W.config5_stream(60, rate_per_s=2000.0, seed=11, max_states=256)
    served = Server(engine).run(stream, realtime=True)
    plain = serve_plain(engine, stream, realtime=True)
    for a, b in zip(served, plain):
        assert_same(norm_gpu(a.result), norm_gpu(b.result), f"request {a.rid}")
    s = summarize(served)
    assert s["p99_ms"] >= s["p50_ms"] > 0


def test_memory_budget_binds_and_results_equal_alone():
    """A budget that holds a few requests at a time: admission defers (several admission calls,
    none over the budget unless a request runs alone), every result equals the request evolved
    alone, and the device footprint the engine reports stays within the estimates admitted.
    Requests over the budget by themselves (uncapped ones) run alone."""
    from hypergraphrewritingengine_b200 import Engine
    from hypergraphrewritingengine_b200.serve import estimate_bytes
    stream = W.config5_stream(24, rate_per_s=1e9, seed=21, max_states=1024)
    # two uncapped requests with a small step budget: estimated past the budget, so alone
    for k in (5, 17):
        t, ev = stream[k]
        stream[k] = (t, W.Evolution(rules=ev.rules, roots=ev.roots, steps=2, max_states=0))
    est = [estimate_bytes(ev) for _, ev in stream]
    capped = sorted(e for (_, ev), e in zip(stream, est) if ev.max_states)
    budget = capped[-1] * 3.5
    assert est[5] > budget and est[17] > budget
    eng = Engine(0)        # a fresh engine: its footprint is this stream's alone
    try:
        srv = Server(eng, memory_budget=budget, track_device_bytes=True)
        recs = srv.run(stream, realtime=False)
        assert len(srv.admit_sizes) > 3 and sum(srv.admit_sizes) == len(stream)
        assert srv.peak_device_bytes <= srv.peak_reserved
        for rec, (_, ev) in zip(recs, stream):
            alone = eng.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(norm_gpu(rec.result), norm_gpu(alone), f"request {rec.rid}")
    finally:
        eng.close()
