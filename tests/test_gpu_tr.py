"""Transitive reduction of the causal graph on the device (HGX_OPT_TRANSITIVE_REDUCTION).

Full multiway against the reference engine's own reduced relation (tests/golden, "tr" section);
WL quotient, caps and batches against the oracle's reduction of its own relation. Exact
comparisons of the causal key multisets (integer work).
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
def tr_engine(engine):
    engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 1)
    try:
        yield engine
    finally:
        engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 0)


@pytest.mark.parametrize("name", sorted(FULL))
def test_reduced_causal_matches_reference(tr_engine, golden, name):
    rules, roots, steps = FULL[name]
    n = norm_gpu(tr_engine.evolve(rules, roots, steps, quotient=False))
    g = golden["tr"][name]
    assert n["causal"] == g["causal"], name
    assert pyoracle.digest(n["causal_keys"]) == g["causal_digest"], name
    # everything but the causal relation is unchanged by the reduction
    full = golden["full"][name]
    assert n["events"] == full["events"] and n["branchial"] == full["branchial"], name


def _oracle_cases():
    out = [W.config2(6), W.config3(5),
           W.Evolution(rules=[cases.C2_RULE], roots=[cases.C2_INIT], steps=6, quotient=True,
                       max_states=300),
           W.Evolution(rules=[cases.C1_RULE], roots=[cases.C1_INIT], steps=5, quotient=False,
                       max_states=2000)]
    for name, rules, init, depth in cases.CORPUS:
        out.append(W.Evolution(rules=rules, roots=[init], steps=depth + 1, quotient=True))
    return out


def test_reduced_causal_matches_oracle(tr_engine):
    for ev in _oracle_cases():
        res = tr_engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                               max_states=ev.max_states)
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                              max_states=ev.max_states, tr=True)
        assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name or ev.steps} tr")


def test_reduced_causal_batch_and_counts(tr_engine):
    evs = W.config4(n=40, max_states=512)
    for ev, res in zip(evs, tr_engine.evolve_batch(evs)):
        ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True,
                              max_states=ev.max_states, tr=True)
        assert_same(norm_gpu(res), norm_oracle(ref), f"{ev.name} tr")
    # device-resident counts agree with the reduced relation
    ev = W.config2(6)
    c = tr_engine.counts(ev.rules, ev.roots, ev.steps, True, ev.max_states)
    ref = pyoracle.evolve(ev.rules, ev.roots, ev.steps, quotient=True, tr=True)
    assert c["causal"] == len(ref["causal"])


def test_reduction_past_64_levels_is_rejected(tr_engine):
    # a rule that applies forever on a one-edge state: 70 levels
    with pytest.raises(api.HgxError):
        tr_engine.evolve([([[0, 1]], [[0, 1]])], [[[1, 2]]], 70, quotient=False)
    # the engine is usable afterwards
    res = tr_engine.evolve([cases.C1_RULE], [cases.C1_INIT], 3, quotient=False)
    assert res.num_events > 0
