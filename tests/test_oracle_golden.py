"""The oracle (CPU restatement) pinned against the reference engine's own outputs.

Runs on CPU only. The fixtures in tests/golden/golden.json were produced by the reference CPU
engine compiled from its own sources (oracle/_ref, see tests/golden/make_golden.py).
"""
import random

import numpy as np
import pytest

import cases
from oracle import pyoracle
from parity import assert_matches_golden, norm_oracle


def _case_table(kind):
    src = cases.all_full_cases() if kind == "full" else cases.all_quotient_cases()
    return {name: (rules, roots, steps) for name, rules, roots, steps in src}


FULL = _case_table("full")
QUOT = _case_table("quotient")


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_multiway_matches_reference(name, golden):
    rules, roots, steps = FULL[name]
    r = pyoracle.evolve(rules, roots, steps, quotient=False)
    assert_matches_golden(norm_oracle(r), golden["full"][name], name)


@pytest.mark.parametrize("name", sorted(FULL))
def test_transitive_reduction_matches_reference(name, golden):
    """Causal graph with transitive reduction on (the reference's product default)."""
    rules, roots, steps = FULL[name]
    r = pyoracle.evolve(rules, roots, steps, quotient=False, tr=True)
    n = norm_oracle(r)
    g = golden["tr"][name]
    assert n["causal"] == g["causal"], name
    assert pyoracle.digest(n["causal_keys"]) == g["causal_digest"], name
    if "causal_keys" in g:
        assert np.array_equal(n["causal_keys"], np.array(g["causal_keys"], np.uint64)), name


@pytest.mark.parametrize("keys", [3, 15])
@pytest.mark.parametrize("name", sorted(FULL))
def test_event_canonicalisation_matches_reference(name, keys, golden):
    """Canonical event count under event signature keys. The reference hashes states exactly (IR)
    once event keys are on; where its class count equals the WL class count the two partitions
    coincide (isomorphic states share a WL hash), so the canonical event counts must agree."""
    rules, roots, steps = FULL[name]
    r = pyoracle.evolve(rules, roots, steps, quotient=False)
    sig = pyoracle.event_signatures(r["state_hash"], r["state_depth"], r["events"], keys)
    g = golden["evsig"][name][str(keys)]
    assert g["raw_events"] == len(r["events"]), name
    n = len(np.unique(sig))
    if g["classes"] == golden["full"][name]["wl_classes"]:
        assert n == g["events"], name
    else:   # WL merged some IR classes: signatures can only merge further
        assert n <= g["events"], name


# WL classes the reference's IR-keyed quotient separates but the WL hash merges (a WL collision
# at the deepest level). Events are unaffected: they come from the levels above.
WL_COLLISIONS = {"c2-quot-5": 3, "c3-quot-5": 1}


@pytest.mark.parametrize("name", sorted(QUOT))
def test_quotient_counts_match_reference(name, golden):
    rules, roots, steps = QUOT[name]
    r = pyoracle.evolve(rules, roots, steps, quotient=True)
    g = golden["quotient"][name]
    assert len(r["events"]) == g["events"], name
    assert r["classes"] == g["ir_classes"] - WL_COLLISIONS.get(name, 0), name


def test_golden_matrix_rows(golden):
    """The reference's cached golden matrix (None/None/full multiway rows): event counts."""
    corpus = {name: (rules, init) for name, rules, init, _ in cases.CORPUS}
    checked = 0
    for name, row in golden["matrix"].items():
        if name not in corpus:
            continue
        rules, init = corpus[name]
        r = pyoracle.evolve(rules, [init], row["steps"], quotient=False)
        assert len(r["events"]) == row["events"], name
        assert len(r["state_hash"]) == row["states"], name
        checked += 1
    assert checked >= 15


@pytest.mark.parametrize("name,steps", [("c2", 5), ("c3", 4)])
def test_quotient_classes_are_full_multiway_classes(name, steps):
    """Each WL class the quotient finds is a WL class of the full unfolding, and without WL
    collisions they are the same set (shortest-depth expansion reaches every class)."""
    rule, init = {"c2": (cases.C2_RULE, cases.C2_INIT), "c3": (cases.C3_RULE, cases.C3_INIT)}[name]
    f = pyoracle.evolve([rule], [init], steps, quotient=False)
    q = pyoracle.evolve([rule], [init], steps, quotient=True)
    assert set(np.unique(q["state_hash"]).tolist()) == set(np.unique(f["state_hash"]).tolist())


def _random_state(rng, n_edges, n_verts, arities=(2, 3)):
    return [[rng.randint(1, n_verts) for _ in range(rng.choice(arities))] for _ in range(n_edges)]


def test_wl_hash_is_label_and_order_invariant():
    rng = random.Random(7)
    for _ in range(200):
        st = _random_state(rng, rng.randint(1, 24), rng.randint(2, 16), arities=(2, 3, 4))
        h = pyoracle.wl_hash(st)
        perm = list(range(1, 40))
        rng.shuffle(perm)
        relabeled = [[perm[v] for v in e] for e in st]
        shuffled = relabeled[:]
        rng.shuffle(shuffled)
        assert pyoracle.wl_hash(relabeled) == h
        assert pyoracle.wl_hash(shuffled) == h


def test_wl_hash_empty_state_is_reserved():
    assert pyoracle.wl_hash([]) == 0x9E3779B97F4A7C15


def test_state_cap_truncates_at_first_excess_event():
    rules, roots = [cases.C2_RULE], [cases.C2_INIT]
    full = pyoracle.evolve(rules, roots, 5, quotient=True)
    capped = pyoracle.evolve(rules, roots, 5, quotient=True, max_states=100)
    assert capped["truncated"] and not full["truncated"]
    assert capped["classes"] == 100
    # the capped run is a prefix of the uncapped one in canonical event order
    n = len(capped["events"])
    assert np.array_equal(capped["events"][:, 2:], full["events"][:n, 2:])


def _corpus():
    import json
    import os
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_corpus.json")
    return json.load(open(p))["cases"]


def test_oracle_matches_reference_golden_corpus():
    """The reference's shared engine corpus (reference/golden_corpus.wl, 12 MultiwaySystem cases
    in full multiway): classes, raw events, causal pairs of the transitively reduced relation and
    branchial pairs, all equal (WL classes coincide with the IR classes on every case)."""
    import numpy as np
    for c in _corpus():
        r = pyoracle.evolve(c["rules"], [c["init"]], c["steps"], quotient=False, tr=True)
        got = {"states": len(np.unique(r["state_hash"])), "raw_events": len(r["events"]),
               "causal": len({(int(a), int(b)) for a, b, _ in r["causal"]}),
               "branchial": len(r["branchial"])}
        assert got == c["expected"], c["name"]
