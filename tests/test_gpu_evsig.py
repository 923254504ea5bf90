"""Event canonicalisation on the device (HGX_OPT_EVENT_SIGNATURE_KEYS): signatures over the WL
hashes, the canonical event count, and causal/branchial unchanged. Against the oracle on every
case (exact signature multisets) and, through the oracle's pinning, the reference's canonical
event counts. Integer work: exact comparisons.
"""
import numpy as np
import pytest

import cases
from hypergraphrewritingengine_b200 import api
from hypergraphrewritingengine_b200 import workloads as W
from oracle import pyoracle
from parity import assert_same, norm_gpu, norm_oracle

pytestmark = pytest.mark.gpu

FULL = {name: (rules, roots, steps) for name, rules, roots, steps in cases.all_full_cases()}


@pytest.fixture
def keyed(engine):
    yield engine
    engine.set_option(api.OPT_EVENT_SIGNATURE_KEYS, 0)


def _check(res, ref, keys, what):
    want = pyoracle.event_signatures(ref["state_hash"], ref["state_depth"], ref["events"], keys)
    got = np.asarray(res.event_signature, dtype=np.uint64)
    assert len(got) == res.num_events, what
    assert np.array_equal(np.sort(got), np.sort(want)), what
    assert res.num_canonical_events == len(np.unique(want)), what
    # the canonical event of a signature is its first event
    canon = res.canonical_event()
    assert all(got[canon[i]] == got[i] and canon[i] <= i for i in range(0, len(got), 97)), what
    # the relations are over every application, as in the reference
    assert_same(norm_gpu(res), norm_oracle(ref), what)


@pytest.mark.parametrize("keys", [3, 15])
@pytest.mark.parametrize("name", sorted(FULL))
def test_full_multiway_signatures(keyed, golden, name, keys):
    rules, roots, steps = FULL[name]
    keyed.set_option(api.OPT_EVENT_SIGNATURE_KEYS, keys)
    res = keyed.evolve(rules, roots, steps, quotient=False)
    _check(res, pyoracle.evolve(rules, roots, steps, quotient=False), keys, f"{name}/{keys}")
    g = golden["evsig"][name][str(keys)]
    if g["classes"] == golden["full"][name]["wl_classes"]:
        assert res.num_canonical_events == g["events"], name


@pytest.mark.parametrize("keys", [1, 2, 3, 6, 15])
def test_quotient_batch_and_counts(keyed, keys):
    keyed.set_option(api.OPT_EVENT_SIGNATURE_KEYS, keys)
    for ev in (W.config2(6), W.config3(5)):
        res = keyed.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        _check(res, ref, keys, f"{ev.name}/{keys}")
        c = keyed.counts(ev.rules, ev.roots, ev.steps, True, ev.max_states)
        assert c["canonical_events"] == res.num_canonical_events
    evs = W.config4(n=24, max_states=512)
    for ev, res in zip(evs, keyed.evolve_batch(evs)):
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        _check(res, ref, keys, f"{ev.name}/{keys}")


def test_off_and_rejected_keys(keyed):
    res = keyed.evolve([cases.C1_RULE], [cases.C1_INIT], 3, quotient=False)
    assert len(res.event_signature) == 0 and res.num_canonical_events == res.num_events
    for bad in (16, 32, 0x3F):
        with pytest.raises(api.HgxError):
            keyed.set_option(api.OPT_EVENT_SIGNATURE_KEYS, bad)


def test_reference_shaped_api_event_keys():
    hg = api.Hypergraph()
    hg.set_event_signature_keys(api.EVENT_SIG_FULL)
    eng = api.ParallelEvolutionEngine(hg, 8)
    eng.add_rule(api.make_rule(0).lhs([0, 1]).lhs([1, 2]).rhs([0, 1]).rhs([1, 2]).rhs([2, 0]).build())
    eng.evolve([[1, 2], [2, 3], [3, 1]], 5)
    assert hg.num_events() == 33          # the reference engine's canonical event count
    assert hg.num_raw_events() == 22203
    with pytest.raises(ValueError):
        hg.set_event_signature_keys(0x30)


def test_served_signatures(keyed):
    """Finished requests finalised on the device carry the same signatures."""
    from hypergraphrewritingengine_b200.serve import Server
    keyed.set_option(api.OPT_EVENT_SIGNATURE_KEYS, 15)
    stream = W.config5_stream(12, rate_per_s=1000.0, seed=5, max_states=256)
    for rec, (_, ev) in zip(Server(keyed).run(stream, realtime=False, admit_per_step=3), stream):
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        _check(rec.result, ref, 15, f"request {rec.rid}")
