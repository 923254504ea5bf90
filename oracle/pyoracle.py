"""Python side of the oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (the C++ restatement in ``restate.cpp``) through ctypes and
provides the result normalisation that both the oracle's and the CUDA path's results go
through before they are compared.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s ``cpu_baseline`` leg import this module; the product library never does.

Normalisation follows the reference's own cross-engine comparison
(gpu/tests/test_gpu_vs_cpu_differential.cpp:119-157):
  * event key      fnv(fnv(fnv(fnv(OFFSET, hash(in)), hash(out)), rule), step)
  * causal key     fnv(fnv(OFFSET, key(producer)), key(consumer))         (directed)
  * branchial key  fnv(fnv(OFFSET, min(key a, key b)), max(key a, key b))  (unordered)
Each multiset is compared sorted, or through ``digest`` (an FNV fold of the sorted array and
its length), which is what the committed golden fixtures store for the large cases.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "hgref")

FNV_OFFSET = np.uint64(0xCBF29CE484222325)
FNV_PRIME = np.uint64(0x100000001B3)


def _fold(h, x):
    with np.errstate(over="ignore"):
        return (np.bitwise_xor(h, x)) * FNV_PRIME


def event_keys(in_hash, out_hash, rule, step):
    h = np.full(len(in_hash), FNV_OFFSET, dtype=np.uint64)
    h = _fold(h, np.asarray(in_hash, dtype=np.uint64))
    h = _fold(h, np.asarray(out_hash, dtype=np.uint64))
    h = _fold(h, np.asarray(rule, dtype=np.uint64))
    h = _fold(h, np.asarray(step, dtype=np.uint64))
    return h


def event_signatures(state_hash, state_depth, events, keys):
    """Per event, hgcommon::event_signature (common/include/hgcommon/event_core.hpp:64-84) over
    the WL hashes: keys bit 0 input state, 1 output state, 2 step, 3 rule, folded in that order;
    0 and the bare offset map to 1. The step is that of the output's canonical state, the first
    state created with its hash (Hypergraph::get_canonical_state_for_event,
    hypergraph/src/hypergraph.cpp:362-377, read at :486-490): the class's smallest depth.
    events: uint32 [n, 4] = (in, out, rule, step)."""
    sh = np.asarray(state_hash, dtype=np.uint64)
    sd = np.asarray(state_depth, dtype=np.uint64)
    ev = np.asarray(events, dtype=np.uint32).reshape(-1, 4)
    sig = np.full(len(ev), FNV_OFFSET, dtype=np.uint64)
    if keys & 1:
        sig = _fold(sig, sh[ev[:, 0]])
    if keys & 2:
        sig = _fold(sig, sh[ev[:, 1]])
    if keys & 4:
        first_depth = {}
        for h, d in zip(sh.tolist(), sd.tolist()):
            if d < first_depth.get(h, 1 << 62):
                first_depth[h] = d
        step = np.array([first_depth[h] for h in sh[ev[:, 1]].tolist()], dtype=np.uint64)
        sig = _fold(sig, step)
    if keys & 8:
        sig = _fold(sig, ev[:, 2].astype(np.uint64))
    sig[(sig == 0) | (sig == FNV_OFFSET)] = np.uint64(1)
    return sig


def directed_pair_keys(a, b):
    h = np.full(len(a), FNV_OFFSET, dtype=np.uint64)
    return _fold(_fold(h, np.asarray(a, dtype=np.uint64)), np.asarray(b, dtype=np.uint64))


def unordered_pair_keys(a, b):
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    return directed_pair_keys(np.minimum(a, b), np.maximum(a, b))


def digest(values) -> int:
    """FNV fold of a sorted uint64 array followed by its length (matches ref_harness.cpp)."""
    v = np.sort(np.asarray(values, dtype=np.uint64))
    h = int(FNV_OFFSET)
    p = int(FNV_PRIME)
    mask = (1 << 64) - 1
    # Python ints: exact and fast enough for the fixture sizes used here (<= a few 1e5).
    for x in v.tolist():
        h = ((h ^ x) * p) & mask
    return ((h ^ len(v)) * p) & mask


def normalize(state_hash, events, causal, branchial):
    """Normalise a raw result.

    state_hash: uint64 [n_states]; events: uint32 [n_events, 4] = (in, out, rule, step);
    causal: uint32 [n, >=2] (producer, consumer, ...); branchial: uint32 [n, 2].
    Returns a dict of counts and sorted key arrays.
    """
    state_hash = np.asarray(state_hash, dtype=np.uint64)
    events = np.asarray(events, dtype=np.uint32).reshape(-1, 4)
    ek = event_keys(state_hash[events[:, 0]], state_hash[events[:, 1]], events[:, 2], events[:, 3])
    causal = np.asarray(causal, dtype=np.uint32).reshape(len(causal), -1) if len(causal) else np.zeros((0, 3), np.uint32)
    branchial = np.asarray(branchial, dtype=np.uint32).reshape(-1, 2)
    ck = directed_pair_keys(ek[causal[:, 0]], ek[causal[:, 1]]) if len(causal) else np.zeros(0, np.uint64)
    bk = unordered_pair_keys(ek[branchial[:, 0]], ek[branchial[:, 1]]) if len(branchial) else np.zeros(0, np.uint64)
    classes = np.unique(state_hash)
    return {
        "raw_states": int(len(state_hash)),
        "wl_classes": int(len(classes)),
        "events": int(len(events)),
        "causal": int(len(ck)),
        "branchial": int(len(bk)),
        "state_hashes": classes,
        "event_keys": np.sort(ek),
        "causal_keys": np.sort(ck),
        "branchial_keys": np.sort(bk),
    }


# --------------------------------------------------------------------------------------------
# Blob encoding shared with the product C-ABI (include/hgx.h).
# --------------------------------------------------------------------------------------------

def encode_rules(rules):
    """rules: list of (lhs_edges, rhs_edges), each a list of lists of variable indices."""
    out = [len(rules)]
    for lhs, rhs in rules:
        for side in (lhs, rhs):
            out.append(len(side))
            for e in side:
                out.append(len(e))
                out.extend(int(v) for v in e)
    return np.asarray(out, dtype=np.uint32)


def encode_roots(roots):
    """roots: list of states, each a list of edges (lists of vertex ids)."""
    out = [len(roots)]
    for st in roots:
        out.append(len(st))
        for e in st:
            out.append(len(e))
            out.extend(int(v) for v in e)
    return np.asarray(out, dtype=np.uint32)


# --------------------------------------------------------------------------------------------
# The restatement (liboracle.so)
# --------------------------------------------------------------------------------------------

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.oracle_wl_hash.argtypes = [u32p, ctypes.c_size_t]
        L.oracle_wl_hash.restype = ctypes.c_uint64
        L.oracle_evolve.argtypes = [u32p, ctypes.c_size_t, u32p, ctypes.c_size_t, ctypes.c_uint32,
                                    ctypes.c_int, ctypes.c_uint64]
        L.oracle_evolve.restype = ctypes.c_void_p
        L.oracle_count.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_count.restype = ctypes.c_uint64
        L.oracle_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_copy.restype = None
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_free.restype = None
        L.oracle_reduce_causal.argtypes = [ctypes.c_void_p]
        L.oracle_reduce_causal.restype = None
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def wl_hash(edges) -> int:
    blob = [len(edges)]
    for e in edges:
        blob.append(len(e))
        blob.extend(int(v) for v in e)
    b = np.asarray(blob, dtype=np.uint32)
    return int(lib().oracle_wl_hash(_ptr(b), len(b)))


def evolve(rules, roots, steps, quotient=False, max_states=0, tr=False):
    """Run the restatement. Returns raw arrays (state_hash, state_depth, events, causal,
    branchial) plus counts. tr=True reduces the causal triples transitively."""
    L = lib()
    rb = encode_rules(rules)
    sb = encode_roots(roots)
    h = L.oracle_evolve(_ptr(rb), len(rb), _ptr(sb), len(sb), int(steps), int(bool(quotient)),
                        int(max_states))
    if not h:
        raise ValueError("oracle rejected the rule or root encoding")
    try:
        if tr:
            L.oracle_reduce_causal(h)
        ns, ne, nc, nb = (int(L.oracle_count(h, i)) for i in range(4))
        classes = int(L.oracle_count(h, 4))
        truncated = bool(L.oracle_count(h, 5))
        sh = np.zeros(ns, np.uint64)
        sd = np.zeros(ns, np.uint32)
        ev = np.zeros((ne, 4), np.uint32)
        ca = np.zeros((nc, 3), np.uint32)
        br = np.zeros((nb, 2), np.uint32)
        for what, arr in enumerate((sh, sd, ev, ca, br)):
            if arr.size:
                L.oracle_copy(h, what, arr.ctypes.data_as(ctypes.c_void_p))
    finally:
        L.oracle_free(h)
    return {"state_hash": sh, "state_depth": sd, "events": ev, "causal": ca, "branchial": br,
            "classes": classes, "truncated": truncated}


# --------------------------------------------------------------------------------------------
# The reference engine itself (oracle/_ref/hgref, built from the reference's own sources)
# --------------------------------------------------------------------------------------------

def spec_text(rules, roots, steps, quotient=False, threads=0, arrays=False, tr=False, evkeys=0):
    lines = [f"steps {int(steps)}", f"mode {'quotient' if quotient else 'full'}",
             f"threads {int(threads)}", f"arrays {1 if arrays else 0}", f"tr {1 if tr else 0}",
             f"evkeys {int(evkeys)}"]
    for lhs, rhs in rules:
        parts = ["rule", str(len(lhs))]
        for e in lhs:
            parts += [str(len(e))] + [str(v) for v in e]
        parts.append(str(len(rhs)))
        for e in rhs:
            parts += [str(len(e))] + [str(v) for v in e]
        lines.append(" ".join(parts))
    for st in roots:
        parts = ["root", str(len(st))]
        for e in st:
            parts += [str(len(e))] + [str(v) for v in e]
        lines.append(" ".join(parts))
    return "\n".join(lines) + "\n"


def run_reference(rules, roots, steps, quotient=False, threads=0, arrays=False, timeout=None,
                  tr=False, evkeys=0):
    """Run the compiled reference engine harness; returns its parsed JSON line."""
    import json
    import tempfile

    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    with tempfile.NamedTemporaryFile("w", suffix=".spec", delete=False) as f:
        f.write(spec_text(rules, roots, steps, quotient, threads, arrays, tr, evkeys))
        path = f.name
    try:
        out = subprocess.run([REF_BIN, path], capture_output=True, text=True, check=True,
                             timeout=timeout).stdout
    finally:
        os.unlink(path)
    return json.loads(out.strip().splitlines()[-1])
