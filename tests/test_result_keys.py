"""EvolveResult.keys(), the product's schedule-independent normal form of a result, equals the
oracle's normalisation (the reference's cross-engine keys) on the same arrays. CPU only: the
result object is built from an oracle run."""
import numpy as np

from hypergraphrewritingengine_b200 import workloads as W
from hypergraphrewritingengine_b200.api import EvolveResult
from oracle import pyoracle


def _as_result(r):
    z = np.zeros(0, np.uint32)
    return EvolveResult(state_hash=r["state_hash"], state_depth=r["state_depth"],
                        events=r["events"], causal=r["causal"], branchial=r["branchial"],
                        event_cons_off=z, event_cons=z, event_prod=z.reshape(-1, 2),
                        state_edge_off=z, state_edge_ids=z, state_arity=z, state_vert_off=z,
                        state_verts=z, num_classes=int(r["classes"]), truncated=bool(r["truncated"]))


def test_keys_equal_oracle_normalisation():
    for ev, steps, quotient in ((W.config1(), 4, False), (W.config3(4), 4, True)):
        r = pyoracle.evolve(ev.rules, ev.roots, steps, quotient=quotient)
        k = _as_result(r).keys()
        n = pyoracle.normalize(r["state_hash"], r["events"], r["causal"], r["branchial"])
        for name in ("state_hashes", "event_keys", "causal_keys", "branchial_keys"):
            assert np.array_equal(k[name], n[name]), name


def test_same_as_detects_a_difference():
    ev = W.config1()
    r = pyoracle.evolve(ev.rules, ev.roots, 3, quotient=False)
    a, b = _as_result(r), _as_result(r)
    assert a.same_as(b)
    r2 = dict(r)
    r2["branchial"] = r["branchial"][:-1]
    assert not a.same_as(_as_result(r2))
