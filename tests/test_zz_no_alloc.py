"""The allocation-free entry point hgx_hash_states_noalloc, called through the C-ABI.

It serves callers that cannot call cudaMalloc (code under a runtime that owns the device's
memory, or on a path that cannot take cudaMalloc's implicit synchronisation): they hand in their
own device buffers and the library uses a fixed scratch array instead of allocating. Its results
must equal the allocating evolve entry point's (hgx_evolve with zero steps hashes the roots): WL
hashes bit for bit, and the class of each state = the first state with the same hash. Two calls
in a row, with different inputs, check that the reused scratch is cleared between calls.

This file is collected last so that a failure here cannot stop the rest of the suite.
"""
import ctypes
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _records(states):
    """Engine record layout: edge ids | arities packed 4 per word | vertices."""
    words, offs, ne, nocc = [], [], [], []
    eid = 0
    for st in states:
        offs.append(len(words))
        n = len(st)
        ar = [0] * ((n + 3) // 4)
        for k, e in enumerate(st):
            ar[k // 4] |= len(e) << (8 * (k % 4))
        words += list(range(eid, eid + n)) + ar + [v for e in st for v in e]
        eid += n
        ne.append(n)
        nocc.append(sum(len(e) for e in st))
    return (np.asarray(words, np.uint32), np.asarray(offs, np.uint64), np.asarray(ne, np.uint32),
            np.asarray(nocc, np.uint32))


def _random_states(seed, n):
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        ne = rng.choice([1, 2, 4, 8, 16, 30, 60])
        nv = max(2, ne // 2 + rng.randint(0, 3))
        ar = rng.choice([(2,), (3,), (2, 3), (1, 2)])
        st = [[rng.randint(1, nv) for _ in range(rng.choice(ar))] for _ in range(ne)]
        out.append(st)
    # exact duplicates and relabelled copies, so classes hold several states
    for i in range(0, n // 4):
        perm = list(range(200))
        rng.shuffle(perm)
        out.append([[perm[v] for v in e] for e in out[i]])
    return out


def _noalloc(L, states, nocc_fix=None, expect=0):
    import torch
    words, offs, ne, nocc = _records(states)
    if nocc_fix is not None:
        nocc_fix(words, offs, ne, nocc)
    dev = torch.device("cuda", 0)
    d_words = torch.from_numpy(words.view(np.int32)).to(dev)
    d_offs = torch.from_numpy(offs.view(np.int64)).to(dev)
    d_ne = torch.from_numpy(ne.view(np.int32)).to(dev)
    d_nocc = torch.from_numpy(nocc.view(np.int32)).to(dev)
    d_hash = torch.empty(len(states), dtype=torch.int64, device=dev)
    d_cls = torch.empty(len(states), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = L.hgx_hash_states_noalloc(
        ctypes.c_void_p(d_words.data_ptr()), ctypes.c_void_p(d_offs.data_ptr()),
        ctypes.c_void_p(d_ne.data_ptr()), ctypes.c_void_p(d_nocc.data_ptr()), len(states),
        int(ne.max()), int(nocc.max()), ctypes.c_void_p(d_hash.data_ptr()),
        ctypes.c_void_p(d_cls.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == expect, L.hgx_last_error()
    if expect:
        return None
    return d_hash.cpu().numpy().view(np.uint64), d_cls.cpu().numpy().view(np.uint32)


def _allocating(states):
    from hypergraphrewritingengine_b200 import Engine
    eng = Engine(0)
    try:
        res = eng.evolve([([[0, 1]], [[0, 1]])], states, 0, quotient=False)
    finally:
        eng.close()
    first = {}
    cls = np.array([first.setdefault(int(h), i) for i, h in enumerate(res.state_hash)], np.uint32)
    return res.state_hash, cls, res.num_classes


def test_noalloc_matches_allocating_entry_point_twice():
    from hypergraphrewritingengine_b200 import load_library
    L = load_library()
    for seed, n in ((1, 400), (2, 150)):
        states = _random_states(seed, n)
        want_hash, want_cls, n_classes = _allocating(states)
        got_hash, got_cls = _noalloc(L, states)
        assert np.array_equal(got_hash, want_hash)
        assert np.array_equal(got_cls, want_cls)
        assert len(np.unique(got_cls)) == n_classes


def test_noalloc_rejects_oversize_batch():
    from hypergraphrewritingengine_b200 import load_library
    L = load_library()
    st = L.hgx_hash_states_noalloc(None, None, None, None, (1 << 19) + 1, 4, 8, None, None, None)
    assert st == 3   # HGX_ERR_CAPACITY
    assert b"exceed the maximum" in L.hgx_last_error()


def test_noalloc_rejects_inconsistent_record():
    """A caller-supplied record whose arities do not add up to its occurrence count is reported
    as a typed error (HGX_ERR_CAPACITY) instead of being hashed; the next call works."""
    from hypergraphrewritingengine_b200 import load_library
    L = load_library()
    states = _random_states(3, 40)
    bad = 7

    def overstate(words, offs, ne, nocc):
        # one extra vertex word in the declared count: the arities sum to one less than num_occ
        # (the staged occurrences still hold every offset the arities give, so the record is
        # read in bounds whether or not it is checked)
        nocc[bad] += 1

    _noalloc(L, states, nocc_fix=overstate, expect=3)
    assert b"inconsistent" in L.hgx_last_error()
    want_hash, want_cls, _ = _allocating(states)
    got_hash, got_cls = _noalloc(L, states)
    assert np.array_equal(got_hash, want_hash)
    assert np.array_equal(got_cls, want_cls)
