"""The CUDA path against the reference's shared engine golden corpus (reference/golden_corpus.wl,
fixtures in tests/golden/golden_corpus.json made by tests/golden/make_corpus.py): 12
MultiwaySystem cases in full multiway -- classes, raw events, causal pairs of the transitively
reduced relation, branchial pairs -- through the C-ABI."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "golden_corpus.json")))["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_device_matches_reference_golden_corpus(engine, case):
    from hypergraphrewritingengine_b200 import api
    engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 1)
    try:
        res = engine.evolve(case["rules"], [case["init"]], case["steps"], quotient=False)
    finally:
        engine.set_option(api.OPT_TRANSITIVE_REDUCTION, 0)
    got = {"states": len(np.unique(res.state_hash)), "raw_events": int(res.num_events),
           "causal": len({(int(a), int(b)) for a, b, _ in res.causal}),
           "branchial": int(len(res.branchial))}
    assert got == case["expected"]
