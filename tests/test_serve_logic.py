"""Host logic of the continuous-batching request loop (hypergraphrewritingengine_b200/serve.py),
on the CPU: the engine is a stand-in that advances every admitted evolution by one level per
step, so admission order, the memory budget, per-step admission limits, collection and idle
resets are checked without a GPU. The device side of the same loop is tests/test_gpu_serving.py.
"""
from collections import namedtuple

from hypergraphrewritingengine_b200 import serve
from hypergraphrewritingengine_b200 import workloads as W

FakeResult = namedtuple("FakeResult", "evo num_events num_states")


class FakeEngine:
    """The serving calls of api.Engine over a level counter per admitted evolution."""

    def __init__(self):
        self.active = {}          # evolution id -> levels left
        self.finished = []
        self.next_id = 0
        self.resets = 0
        self.steps = 0
        self.collected = []
        self.admit_calls = []

    def serve_reset(self):
        assert not self.active, "reset while evolutions are running"
        self.resets += 1
        self.next_id = 0          # ids restart, as the engine's do after a reset

    def serve_admit_batch(self, jobs, n=None):
        n = len(jobs) if n is None else n
        self.admit_calls.append(n)
        ids = []
        for i in range(n):
            evo = self.next_id
            self.next_id += 1
            left = int(jobs[i].steps)
            if left == 0:
                self.finished.append(evo)      # nothing to expand: finished at admission
            else:
                self.active[evo] = left
            ids.append(evo)
        return ids

    def serve_step(self):
        assert self.active, "step with nothing admitted"
        self.steps += 1
        for evo in list(self.active):
            self.active[evo] -= 1
            if self.active[evo] == 0:
                del self.active[evo]
                self.finished.append(evo)

    def serve_take_finished(self):
        done, self.finished = self.finished, []
        return done

    def serve_collect_batch(self, ids):
        self.collected += ids
        return [FakeResult(evo, 3, 2) for evo in ids]

    def evolve(self, rules, roots, steps, quotient=True, max_states=0):
        return FakeResult(-1, steps, steps)


def _stream(steps_list, gap=0.0):
    return [(i * gap, W.Evolution(rules=[([[0, 1]], [[0, 1], [1, 2]])], roots=[[[1, 2]]],
                                  steps=s, quotient=True, max_states=1000))
            for i, s in enumerate(steps_list)]


def test_every_request_served_once_and_short_ones_overtake():
    eng = FakeEngine()
    arrivals = _stream([6, 1, 0, 3, 2])
    recs = serve.Server(eng).run(arrivals, realtime=False)
    assert all(r.result is not None and r.finished >= r.admitted >= 0 for r in recs)
    assert sorted(eng.collected) == sorted(set(eng.collected)) and len(eng.collected) == 5
    # everything fits the budget: one admission call, then one step per level of the longest
    assert eng.admit_calls == [5] and eng.steps == 6
    # the one-level request finished before the six-level one admitted with it
    assert recs[1].finished <= recs[0].finished


def test_memory_budget_limits_the_admitted_set():
    eng = FakeEngine()
    arrivals = _stream([2, 2, 2, 2])
    est = serve.estimate_bytes(arrivals[0][1])
    recs = serve.Server(eng, memory_budget=2.5 * est).run(arrivals, realtime=False)
    assert all(r.result is not None for r in recs)
    # two fit the budget at a time: admissions come in pairs as earlier requests finish
    assert eng.admit_calls == [2, 2]


def test_a_request_over_the_budget_runs_alone():
    eng = FakeEngine()
    arrivals = _stream([1, 1])
    est = serve.estimate_bytes(arrivals[0][1])
    recs = serve.Server(eng, memory_budget=0.5 * est).run(arrivals, realtime=False)
    assert all(r.result is not None for r in recs)
    assert eng.admit_calls == [1, 1]   # each admitted only once the engine is empty


def test_admissions_per_step_are_capped():
    eng = FakeEngine()
    recs = serve.Server(eng).run(_stream([3] * 7), realtime=False, admit_per_step=2)
    assert all(r.result is not None for r in recs)
    assert all(n <= 2 for n in eng.admit_calls) and sum(eng.admit_calls) == 7


def test_realtime_stream_resets_when_idle_and_respects_arrivals():
    eng = FakeEngine()
    arrivals = _stream([1, 1, 1], gap=0.03)
    recs = serve.Server(eng).run(arrivals, realtime=True)
    for r, (t_arr, _) in zip(recs, arrivals):
        assert r.admitted >= t_arr - 1e-6 and r.finished >= r.admitted
    # the engine went idle between the spaced arrivals and was reset each time
    assert eng.resets >= 2
    s = serve.summarize(recs)
    assert s["requests"] == 3 and s["events"] == 9 and s["p99_ms"] >= s["p50_ms"] > 0


def test_plain_path_serves_in_order():
    recs = serve.serve_plain(FakeEngine(), _stream([2, 0, 1]), realtime=False)
    assert [r.result.num_events for r in recs] == [2, 0, 1]
    assert all(recs[i].finished <= recs[i + 1].admitted for i in range(2))


def test_admissions_per_step_below_one_are_rejected():
    import pytest
    for bad in (0, -1):
        with pytest.raises(ValueError):
            serve.Server(FakeEngine()).run(_stream([1]), realtime=False, admit_per_step=bad)
