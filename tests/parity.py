"""Comparison helpers shared by the parity tests: normalise an oracle run, a CUDA run, or a
golden fixture to the same key multisets and compare them exactly (integer work: bit-exact)."""
import numpy as np

from oracle import pyoracle


def norm_oracle(r):
    return pyoracle.normalize(r["state_hash"], r["events"], r["causal"], r["branchial"])


def norm_gpu(res):
    return pyoracle.normalize(res.state_hash, res.events, res.causal, res.branchial)


def assert_same(a, b, what=""):
    for k in ("wl_classes", "events", "causal", "branchial"):
        assert a[k] == b[k], f"{what}: {k} {a[k]} != {b[k]}"
    for k in ("state_hashes", "event_keys", "causal_keys", "branchial_keys"):
        assert np.array_equal(a[k], b[k]), f"{what}: {k} differ"


def assert_matches_golden(n, g, what=""):
    """n: normalised result; g: a golden.json 'full' entry produced by the reference engine."""
    assert n["raw_states"] == g["raw_states"], f"{what}: raw states {n['raw_states']} != {g['raw_states']}"
    for k in ("events", "wl_classes", "causal", "branchial"):
        assert n[k] == g[k], f"{what}: {k} {n[k]} != {g[k]}"
    if "state_hashes" in g:
        assert [int(x) for x in n["state_hashes"]] == g["state_hashes"], f"{what}: state hashes"
    assert pyoracle.digest(n["state_hashes"]) == g["state_digest"], f"{what}: state digest"
    assert pyoracle.digest(n["event_keys"]) == g["event_digest"], f"{what}: event keys"
    assert pyoracle.digest(n["causal_keys"]) == g["causal_digest"], f"{what}: causal keys"
    assert pyoracle.digest(n["branchial_keys"]) == g["branchial_digest"], f"{what}: branchial keys"
    for k in ("event_keys", "causal_keys", "branchial_keys"):
        if k in g:
            assert [int(x) for x in n[k]] == g[k], f"{what}: {k}"
