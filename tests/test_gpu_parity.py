"""Parity of the CUDA path (through the C-ABI) with the oracle and the reference's fixtures.

Integer work throughout: every comparison is exact (WL hashes bit for bit, key multisets equal).
"""
import random

import numpy as np
import pytest

import cases
from hypergraphrewritingengine_b200 import workloads as W
from oracle import pyoracle
from parity import assert_matches_golden, assert_same, norm_gpu, norm_oracle

pytestmark = pytest.mark.gpu


def _random_state(rng, n_edges, n_verts, arities):
    return [[rng.randint(1, n_verts) for _ in range(rng.choice(arities))] for _ in range(n_edges)]


def test_root_wl_hashes_match_oracle(engine):
    """steps=0: the device hashes the roots only (several roots per call, uneven sizes)."""
    rng = random.Random(11)
    roots = []
    for i in range(300):
        ne = rng.choice([1, 2, 3, 5, 8, 13, 20, 40, 90, 200])
        roots.append(_random_state(rng, ne, max(2, ne // 2 + rng.randint(0, 4)),
                                   arities=rng.choice([(2,), (3,), (2, 3), (1, 2, 4), (4, 5)])))
    res = engine.evolve([([[0, 1]], [[0, 1]])], roots, 0, quotient=False)
    want = [pyoracle.wl_hash(r) for r in roots]
    assert [int(h) for h in res.state_hash] == want


FULL = {name: (rules, roots, steps) for name, rules, roots, steps in cases.all_full_cases()}


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_multiway_matches_reference_fixtures(engine, golden, name):
    rules, roots, steps = FULL[name]
    res = engine.evolve(rules, roots, steps, quotient=False)
    assert_matches_golden(norm_gpu(res), golden["full"][name], name)


QUOT = {name: (rules, roots, steps) for name, rules, roots, steps in cases.all_quotient_cases()}


@pytest.mark.parametrize("name", sorted(QUOT))
def test_quotient_matches_oracle(engine, name):
    rules, roots, steps = QUOT[name]
    res = engine.evolve(rules, roots, steps, quotient=True)
    ref = pyoracle.evolve(rules, roots, steps, quotient=True)
    assert_same(norm_gpu(res), norm_oracle(ref), name)


@pytest.mark.parametrize("ev", [W.config2(6), W.config2(7), W.config3(5)], ids=lambda e: e.name)
def test_named_quotient_workloads_match_oracle(engine, ev):
    res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
    ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
    assert_same(norm_gpu(res), norm_oracle(ref), ev.name)
    assert res.num_classes == ref["classes"]


def test_state_cap_matches_oracle(engine):
    for cap in (1, 7, 100, 1000):
        res = engine.evolve([cases.C2_RULE], [cases.C2_INIT], 6, quotient=True, max_states=cap)
        ref = pyoracle.evolve([cases.C2_RULE], [cases.C2_INIT], 6, quotient=True, max_states=cap)
        assert res.truncated == ref["truncated"]
        assert_same(norm_gpu(res), norm_oracle(ref), f"cap {cap}")
    for cap in (5, 300):
        res = engine.evolve([cases.C1_RULE], [cases.C1_INIT], 4, quotient=False, max_states=cap)
        ref = pyoracle.evolve([cases.C1_RULE], [cases.C1_INIT], 4, quotient=False, max_states=cap)
        assert_same(norm_gpu(res), norm_oracle(ref), f"full cap {cap}")


def test_batch_matches_single_and_oracle(engine):
    evs = W.config4(n=48, max_states=512)
    batch = engine.evolve_batch(evs)
    for ev, res in zip(evs, batch):
        single = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        a, b, c = norm_gpu(res), norm_gpu(single), norm_oracle(ref)
        assert_same(a, b, ev.name)
        assert_same(a, c, ev.name)
        assert res.truncated == ref["truncated"]


def test_state_edge_records_are_the_oracle_states(engine):
    """Every recorded state's edges hash (on the CPU) to the WL hash the device reported."""
    res = engine.evolve([cases.C3_RULE], [cases.C3_INIT], 4, quotient=True)
    for s in range(0, res.num_states, 7):
        assert pyoracle.wl_hash(res.state_edges(s)) == int(res.state_hash[s])


def test_reference_shaped_api(engine):
    from hypergraphrewritingengine_b200 import Hypergraph, ParallelEvolutionEngine, make_rule
    hg = Hypergraph()
    eng = ParallelEvolutionEngine(hg, 8)
    eng.add_rule(make_rule(0).lhs([0, 1]).lhs([1, 2]).rhs([0, 1]).rhs([1, 2]).rhs([2, 0]).build())
    eng.set_transitive_reduction(False)
    eng.evolve([[1, 2], [2, 3], [3, 1]], 5)
    assert hg.num_states() == 22204
    assert hg.num_events() == 22203
    assert hg.num_canonical_states() == 20
    assert hg.causal_graph().num_causal_edges() == 42816
    assert hg.causal_graph().num_branchial_edges() == 78045


@pytest.mark.parametrize("quotient,rule,init,steps,cap", [
    (True, cases.C2_RULE, cases.C2_INIT, 7, 100_000),      # cut inside a chunked level
    (True, cases.C2_RULE, cases.C2_INIT, 7, 26_700),       # cut right after the previous level
    (False, cases.C1_RULE, cases.C1_INIT, 6, 100_000),     # full multiway: raw-state cap
])
def test_chunked_cap_matches_oracle(engine, quotient, rule, init, steps, cap):
    res = engine.evolve([rule], [init], steps, quotient=quotient, max_states=cap)
    ref = pyoracle.evolve([rule], [init], steps, quotient=quotient, max_states=cap)
    assert res.truncated == ref["truncated"]
    assert_same(norm_gpu(res), norm_oracle(ref), f"cap {cap}")


@pytest.mark.parametrize("ev", [W.config2(8), W.config3(6)], ids=lambda e: e.name)
def test_full_size_workloads_match_oracle(engine, ev):
    """The benchmarked sizes themselves (C2: 8 levels, 2M-state cap; C3: 6 levels)."""
    res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
    ref = _oracle_once(ev)
    assert res.truncated == ref["truncated"]
    assert res.num_classes == ref["classes"]
    assert_same(norm_gpu(res), norm_oracle(ref), ev.name)


_ORACLE_CACHE = {}


def _oracle_once(ev):
    key = ev.name
    if key not in _ORACLE_CACHE:
        _ORACLE_CACHE[key] = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                             max_states=ev.max_states)
    return _ORACLE_CACHE[key]


@pytest.mark.parametrize("mode", [1, 2])
def test_c3_full_size_with_forwarding_matches_oracle(engine, mode):
    """C3 as benchmarked -- ternary rule, 6 levels, WL quotient -- with incremental match
    forwarding on (1: every eligible state; 2: states of at least 48 edges)."""
    from hypergraphrewritingengine_b200 import api
    ev = W.config3(6)
    ref = _oracle_once(ev)
    engine.set_option(api.OPT_FORWARDING, mode)
    try:
        res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
    finally:
        engine.set_option(api.OPT_FORWARDING, 0)
    assert res.truncated == ref["truncated"]
    assert res.num_classes == ref["classes"]
    assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} forwarding={mode}")


def _forwarding_cases():
    out = [(W.config2(6), None), (W.config3(5), None),
           (W.Evolution(rules=[cases.C1_RULE], roots=[cases.C1_INIT], steps=4, quotient=False), None),
           # a hub of 100 edges: delta matches overflow the forwarding buffer (fallback path)
           (W.Evolution(rules=[cases.C2_RULE], roots=[[[1, k] for k in range(2, 102)]], steps=2,
                        max_states=3000), None)]
    for name, rules, init, depth in cases.CORPUS:
        out.append((W.Evolution(rules=rules, roots=[init], steps=depth + 1, quotient=True), name))
    return out


@pytest.mark.parametrize("mode", [1, 0, 2])
def test_forwarding_modes_match_oracle(engine, mode):
    from hypergraphrewritingengine_b200 import api
    engine.set_option(api.OPT_FORWARDING, mode)
    try:
        for ev, name in _forwarding_cases():
            res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                max_states=ev.max_states)
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                  max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"{name or ev.name} forwarding={mode}")
        evs = W.config4(n=32, max_states=1024)   # initial states up to 64 edges
        for ev, res in zip(evs, engine.evolve_batch(evs)):
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} forwarding={mode}")
    finally:
        engine.set_option(api.OPT_FORWARDING, 0)


@pytest.mark.parametrize("chunk_min", [0, 100])
def test_capped_rounds_match_oracle(engine, chunk_min):
    """Capped levels built in rounds that stop at each evolution's cut (forced on small cases):
    batches whose evolutions hit their caps in the same level, and single evolutions."""
    from hypergraphrewritingengine_b200 import api
    engine.set_option(api.OPT_CHUNK_MIN, chunk_min)
    try:
        evs = W.config4(n=48, max_states=256)
        evs += [W.Evolution(rules=[cases.C1_RULE], roots=[cases.C1_INIT], steps=5, quotient=False,
                            max_states=cap) for cap in (40, 333)]
        evs += [W.Evolution(rules=[cases.C2_RULE], roots=[cases.C2_INIT], steps=6, quotient=True,
                            max_states=cap) for cap in (1, 7, 100, 1000)]
        for ev, res in zip(evs, engine.evolve_batch(evs)):
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                  max_states=ev.max_states)
            assert res.truncated == ref["truncated"], ev.name
            assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} chunk_min={chunk_min}")
        for ev in evs[-6:]:
            res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                max_states=ev.max_states)
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                  max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"single {ev.name}")
    finally:
        engine.set_option(api.OPT_CHUNK_MIN, 8192)


@pytest.mark.parametrize("split", [2000, 9000, 1])
def test_level_split_matches_oracle(engine, split):
    """A capped single evolution whose levels are counted and expanded as a frontier prefix and
    then the rest: prefixes that hold the cut, prefixes that end before it (the second range
    runs, and a cut there drops the first range's next frontier), and no split at all."""
    from hypergraphrewritingengine_b200 import api
    engine.set_option(api.OPT_LEVEL_SPLIT, split)
    try:
        for cap in (26_700, 60_000, 100_000, 0):
            res = engine.evolve([cases.C2_RULE], [cases.C2_INIT], 7, quotient=True, max_states=cap)
            ref = pyoracle.evolve([cases.C2_RULE], [cases.C2_INIT], 7, quotient=True, max_states=cap)
            assert res.truncated == ref["truncated"], cap
            assert_same(norm_gpu(res), norm_oracle(ref), f"cap {cap} split {split}")
        res = engine.evolve([cases.C1_RULE], [cases.C1_INIT], 6, quotient=False, max_states=50_000)
        ref = pyoracle.evolve([cases.C1_RULE], [cases.C1_INIT], 6, quotient=False, max_states=50_000)
        assert res.truncated == ref["truncated"]
        assert_same(norm_gpu(res), norm_oracle(ref), f"full cap split {split}")
    finally:
        engine.set_option(api.OPT_LEVEL_SPLIT, 0)


@pytest.mark.parametrize("join", [1, 2])
def test_lane_join_variants_match_oracle(engine, join):
    """Both joins of the small-state expand kernel (the autotuner's choices) give the same result."""
    from hypergraphrewritingengine_b200 import api
    engine.set_option(api.OPT_LANE_JOIN, join)
    try:
        for ev in (W.config2(6), W.config3(5)):
            res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} join={join}")
        evs = W.config4(n=32, max_states=1024)
        for ev, res in zip(evs, engine.evolve_batch(evs)):
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} join={join}")
    finally:
        engine.set_option(api.OPT_LANE_JOIN, 0)


def _large_state_cases():
    """Evolutions whose states pass 64 edges (the join indices apply past 96): served-workload draws
    with large initial states (up to 256 edges, rules with repeated variables among them), a
    100-edge hub, and two disconnected LHS edges (candidates from the signature buckets)."""
    out = []
    for t, ev in W.config5_stream(200, rate_per_s=1e9, seed=0xC0FFEE, max_states=400):
        if ev.meta["n_edges"] > 64:
            out.append(W.Evolution(rules=ev.rules, roots=ev.roots, steps=min(ev.steps, 3),
                                   max_states=400, name=f"large-{ev.name}"))
    out.append(W.Evolution(rules=[cases.C2_RULE], roots=[[[1, k] for k in range(2, 102)]], steps=2,
                           max_states=3000, name="hub-100"))
    out.append(W.Evolution(rules=[([[0, 0, 1], [2, 3, 3]], [[0, 1, 4], [2, 3, 4], [4, 4, 0]])],
                           roots=[[[k % 23 + 1, k % 23 + 1, k % 7 + 30] if k % 3 == 0 else
                                   [k % 11 + 1, k % 13 + 40, k % 13 + 40] for k in range(120)]],
                           steps=2, max_states=2000, name="disconnected-lhs"))
    return out


@pytest.mark.parametrize("index", [1, 0])
def test_join_index_modes_match_oracle(engine, index):
    """The join with and without the vertex / signature indices (states past 96 edges) gives the
    oracle's result, alone and in a batch, with and without match forwarding."""
    from hypergraphrewritingengine_b200 import api
    evs = _large_state_cases()
    assert len(evs) >= 8
    engine.set_option(api.OPT_JOIN_INDEX, index)
    try:
        for fwd in (0, 1):
            engine.set_option(api.OPT_FORWARDING, fwd)
            for ev, res in zip(evs, engine.evolve_batch(evs)):
                ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
                assert res.truncated == ref["truncated"], ev.name
                assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} index={index} fwd={fwd}")
        engine.set_option(api.OPT_FORWARDING, 0)
        for ev in evs[-2:]:
            res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            assert_same(norm_gpu(res), norm_oracle(ref), f"single {ev.name} index={index}")
    finally:
        engine.set_option(api.OPT_FORWARDING, 0)
        engine.set_option(api.OPT_JOIN_INDEX, 1)


def test_state_edge_ids_optional(engine):
    """HGX_OPT_KEEP_STATE_EDGE_IDS = 0 leaves the global edge ids out of the state records (the
    reference's default, edge_identity false); everything else is unchanged, alone and batched."""
    import numpy as np
    from hypergraphrewritingengine_b200 import api
    ev = W.config2(5)
    evs = W.config4(n=12, max_states=256)
    full = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True)
    full_b = engine.evolve_batch(evs)
    engine.set_option(api.OPT_KEEP_STATE_EDGE_IDS, 0)
    try:
        slim = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=True)
        slim_b = engine.evolve_batch(evs)
    finally:
        engine.set_option(api.OPT_KEEP_STATE_EDGE_IDS, 1)
    for a, b in [(full, slim)] + list(zip(full_b, slim_b)):
        assert len(b.state_edge_ids) == 0 and len(a.state_edge_ids) == len(a.state_arity)
        for f in ("state_hash", "events", "causal", "branchial", "state_edge_off", "state_arity",
                  "state_vert_off", "state_verts"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
        assert all(a.state_edges(s) == b.state_edges(s) for s in range(0, a.num_states, 97))
        assert b.bytes() < a.bytes()


_RESULT_FIELDS = ("state_hash", "state_depth", "events", "causal", "branchial", "event_cons_off",
                  "event_cons", "event_prod", "state_edge_off", "state_edge_ids", "state_arity",
                  "state_vert_off", "state_verts")


def test_streamed_result_matches_whole(engine):
    """A single evolution's result copied out range by range while the run continues
    (HGX_OPT_STREAM_RESULT) is array for array the result copied whole after the run: capped
    (the cut level split into parts) and uncapped, quotient and full multiway, with each record
    option off in turn. The second streamed call of each runs with the room the first left."""
    import numpy as np
    from hypergraphrewritingengine_b200 import api
    cases_ = [
        (W.config2(8), {}),
        (W.config2(6), {}),
        (W.Evolution(rules=[cases.C2_RULE], roots=[cases.C2_INIT], steps=7, max_states=26_700), {}),
        (W.config3(5), {}),
        (W.Evolution(rules=[cases.C1_RULE], roots=[cases.C1_INIT], steps=5, quotient=False), {}),
        (W.Evolution(rules=[([[0, 1], [0, 1], [1, 2]], [[0, 1], [1, 2], [1, 2], [2, 3]])],
                     roots=[[[1, 2]] * 4 + [[2, 3]] * 3 + [[2, 2], [3, 1]]], steps=4, max_states=20_000,
                     name="twin-pairs"), {}),
        (W.config2(6), {api.OPT_RECORD_CAUSAL: 0}),
        (W.config2(6), {api.OPT_RECORD_BRANCHIAL: 0}),
        (W.config2(6), {api.OPT_KEEP_STATE_EDGE_IDS: 0}),
        (W.config2(6), {api.OPT_KEEP_STATE_EDGES: 0}),
        (W.Evolution(rules=[cases.C2_RULE], roots=[cases.C2_INIT], steps=0), {}),
    ]
    defaults = {api.OPT_RECORD_CAUSAL: 1, api.OPT_RECORD_BRANCHIAL: 1, api.OPT_KEEP_STATE_EDGE_IDS: 1,
                api.OPT_KEEP_STATE_EDGES: 1}
    streamed_any = 0
    try:
        for ev, opts in cases_:
            for k, v in opts.items():
                engine.set_option(k, v)
            engine.set_option(api.OPT_STREAM_RESULT, 0)
            whole = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
            assert not engine.result_stats()["streamed"]
            engine.set_option(api.OPT_STREAM_RESULT, 2)   # whatever the result's size
            for rep in range(2):
                res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
                st = engine.result_stats()
                streamed_any += st["streamed"]
                if rep == 1 and ev.steps > 0:
                    assert st["streamed"], f"{ev.name} {opts}: second call not streamed"
                for f in _RESULT_FIELDS:
                    a, b = getattr(res, f), getattr(whole, f)
                    assert a.dtype == b.dtype and np.array_equal(a, b), f"{ev.name} {opts} rep {rep}: {f}"
                assert (res.num_states, res.num_events, res.num_classes, res.truncated) == \
                    (whole.num_states, whole.num_events, whole.num_classes, whole.truncated)
            for k in opts:
                engine.set_option(k, defaults[k])
        assert streamed_any >= 10
    finally:
        engine.set_option(api.OPT_STREAM_RESULT, 1)
        for k, v in defaults.items():
            engine.set_option(k, v)


def test_counts_only_causal_matches_result(engine):
    """The causal triples counted on the device level by level (results left on the device)
    equal the triples of the result read back: quotient and full multiway, capped, with and
    without transitive reduction, alone and batched."""
    from hypergraphrewritingengine_b200 import api
    evs = [W.config2(6), W.config3(5), W.config1(),
           W.Evolution(rules=[cases.C2_RULE], roots=[cases.C2_INIT], steps=7, max_states=26_700)]
    try:
        for tr in (0, 1):
            engine.set_option(api.OPT_TRANSITIVE_REDUCTION, tr)
            for ev in evs:
                res = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
                c = engine.counts(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
                assert c["causal"] == len(res.causal), (ev.name, tr)
                assert c["events"] == res.num_events and c["branchial"] == len(res.branchial), (ev.name, tr)
        engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 0)
        batch = W.config4(n=24, max_states=1024)
        results = engine.evolve_batch(batch)
        jobs, _keep = engine.make_jobs(batch)
        outs = (api.ctypes.c_void_p * len(batch))()
        engine.set_option(api.OPT_READBACK, 0)
        try:
            api._check(engine._L.hgx_evolve_batch(engine._h, jobs, len(batch), outs))
        finally:
            engine.set_option(api.OPT_READBACK, 1)
        try:
            for i, (ev, r) in enumerate(zip(batch, results)):
                assert int(engine._L.hgx_result_count(outs[i], api.COUNT_CAUSAL)) == len(r.causal), ev.name
                assert int(engine._L.hgx_result_count(outs[i], api.COUNT_EVENTS)) == r.num_events, ev.name
        finally:
            for i in range(len(batch)):
                engine._L.hgx_result_free(outs[i])
    finally:
        engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 0)


def test_streamed_result_outgrowing_its_blocks(engine):
    """A result larger than the page-locked blocks its engine's previous result sized is not
    streamed: it is finalised whole after the run and equals the unstreamed result; the call
    after it streams into blocks of its own size."""
    import numpy as np
    from hypergraphrewritingengine_b200 import api
    small, big = W.config2(4), W.config2(6)
    try:
        engine.set_option(api.OPT_STREAM_RESULT, 0)
        whole = engine.evolve(big.rules, big.roots, big.steps, quotient=True)
        engine.set_option(api.OPT_STREAM_RESULT, 2)
        engine.evolve(small.rules, small.roots, small.steps, quotient=True)
        engine.evolve(small.rules, small.roots, small.steps, quotient=True)
        assert engine.result_stats()["streamed"]
        first = engine.evolve(big.rules, big.roots, big.steps, quotient=True)
        assert not engine.result_stats()["streamed"]
        second = engine.evolve(big.rules, big.roots, big.steps, quotient=True)
        assert engine.result_stats()["streamed"]
        for res in (first, second):
            for f in _RESULT_FIELDS:
                assert np.array_equal(getattr(res, f), getattr(whole, f)), f
    finally:
        engine.set_option(api.OPT_STREAM_RESULT, 1)
