"""ctypes binding of ``libhgx.so`` (include/hgx.h) and the reference-shaped Python API.

Two layers:

* ``Engine`` -- thin wrapper of the C-ABI: ``evolve``, ``evolve_batch`` and the serving calls,
  returning results as numpy arrays (``EvolveResult``).
* ``make_rule`` / ``RuleBuilder`` / ``Hypergraph`` / ``ParallelEvolutionEngine`` -- the same
  surface as the reference C++ engine API (hypergraph/include/hypergraph/pattern.hpp:142-213,
  parallel_evolution.hpp:743-1041, hypergraph.hpp:567-811), so a caller of the reference can
  switch with the same call sequence:

      hg = Hypergraph()
      engine = ParallelEvolutionEngine(hg)
      engine.add_rule(make_rule(0).lhs([0, 1]).lhs([1, 2]).rhs([0, 1]).rhs([1, 2]).rhs([2, 0]).build())
      engine.set_transitive_reduction(False)
      engine.evolve([[1, 2], [2, 3], [3, 1]], 5)
      hg.num_states(), hg.num_events(), hg.num_canonical_states()

The CUDA library is required: there is no CPU fallback, and every call fails loudly (OSError
or HgxError) when the library or a device is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# HGX_LIB names another build of the library (for comparing builds side by side)
LIB_PATH = os.environ.get("HGX_LIB", os.path.join(HERE, "libhgx.so"))

HGX_OK, HGX_ERR_INVALID, HGX_ERR_CUDA, HGX_ERR_CAPACITY, HGX_ERR_NO_DEVICE, HGX_ERR_INTERNAL = range(6)
(OPT_QUOTIENT, OPT_MAX_STATES, OPT_TRANSITIVE_REDUCTION, OPT_RECORD_CAUSAL, OPT_RECORD_BRANCHIAL,
 OPT_KEEP_STATE_EDGES, OPT_TIMING, OPT_READBACK, OPT_FORWARDING, OPT_CHUNK_MIN,
 OPT_EVENT_SIGNATURE_KEYS, OPT_LANE_JOIN, OPT_LEVEL_SPLIT, OPT_MAX_DEVICE_BYTES,
 OPT_JOIN_INDEX, OPT_KEEP_STATE_EDGE_IDS, OPT_STREAM_RESULT) = range(17)
(COUNT_STATES, COUNT_EVENTS, COUNT_CLASSES, COUNT_CAUSAL, COUNT_BRANCHIAL, COUNT_TRUNCATED,
 COUNT_CONSUMED, COUNT_STATE_EDGES, COUNT_STATE_VERTS, COUNT_RAW_STATES,
 COUNT_CANONICAL_EVENTS) = range(11)
(ARR_STATE_HASH, ARR_STATE_DEPTH, ARR_EVENTS, ARR_CAUSAL, ARR_BRANCHIAL, ARR_EVENT_CONS_OFF,
 ARR_EVENT_CONS, ARR_EVENT_PROD, ARR_STATE_EDGE_OFF, ARR_STATE_EDGE_IDS, ARR_STATE_ARITY,
 ARR_STATE_VERT_OFF, ARR_STATE_VERTS, ARR_EVENT_SIG) = range(14)
# hgcommon EventSignatureKeys bits provided on this path; FULL is the reference's Full preset
EVENT_KEY_INPUT, EVENT_KEY_OUTPUT, EVENT_KEY_STEP, EVENT_KEY_RULE = 1, 2, 4, 8
EVENT_SIG_NONE, EVENT_SIG_FULL = 0, 3

_FNV_OFFSET = np.uint64(0xCBF29CE484222325)
_FNV_PRIME = np.uint64(0x100000001B3)

# Every symbol include/hgx.h declares (the library must export all of them).
EXPORTS = (
    "hgx_last_error", "hgx_version", "hgx_engine_create", "hgx_engine_destroy",
    "hgx_engine_add_rule", "hgx_engine_clear_rules", "hgx_engine_set_option", "hgx_evolve",
    "hgx_evolve_batch", "hgx_serve_reset", "hgx_serve_admit", "hgx_serve_admit_batch", "hgx_serve_step",
    "hgx_serve_take_finished", "hgx_serve_collect", "hgx_serve_collect_batch", "hgx_serve_device_bytes",
    "hgx_result_count",
    "hgx_result_copy", "hgx_result_free", "hgx_engine_stage_times", "hgx_engine_expand_stats", "hgx_engine_result_stats",
    "hgx_engine_stream", "hgx_hash_states_noalloc", "hgx_result_view",
    "hgx_estimate_device_bytes", "hgx_device_memory", "hgx_result_views",
)


class HgxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"hgx status {status}: {message}")
        self.status = status


class Job(ctypes.Structure):
    _fields_ = [("rules", ctypes.POINTER(ctypes.c_uint32)), ("rules_len", ctypes.c_size_t),
                ("roots", ctypes.POINTER(ctypes.c_uint32)), ("roots_len", ctypes.c_size_t),
                ("steps", ctypes.c_uint32), ("quotient", ctypes.c_uint32),
                ("max_states", ctypes.c_uint64)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libhgx.so (raises OSError if it is missing -- build it with build.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build the CUDA library first "
                      "(python -m hypergraphrewritingengine_b200.build)")
    L = ctypes.CDLL(path)
    vp, u32p, u64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)
    sig = {
        "hgx_last_error": ([], ctypes.c_char_p),
        "hgx_version": ([], ctypes.c_char_p),
        "hgx_engine_create": ([ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_engine_destroy": ([vp], None),
        "hgx_engine_add_rule": ([vp, u32p, ctypes.c_size_t], ctypes.c_int),
        "hgx_engine_clear_rules": ([vp], ctypes.c_int),
        "hgx_engine_set_option": ([vp, ctypes.c_int, ctypes.c_uint64], ctypes.c_int),
        "hgx_evolve": ([vp, u32p, ctypes.c_size_t, ctypes.c_uint32, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_evolve_batch": ([vp, ctypes.POINTER(Job), ctypes.c_uint32, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_serve_reset": ([vp], ctypes.c_int),
        "hgx_serve_admit": ([vp, ctypes.POINTER(Job), u32p], ctypes.c_int),
        "hgx_serve_admit_batch": ([vp, ctypes.POINTER(Job), ctypes.c_uint32, u32p], ctypes.c_int),
        "hgx_serve_step": ([vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "hgx_serve_take_finished": ([vp, u32p, ctypes.c_uint32, u32p], ctypes.c_int),
        "hgx_serve_collect": ([vp, ctypes.c_uint32, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_serve_collect_batch": ([vp, u32p, ctypes.c_uint32, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_serve_device_bytes": ([vp, u64p], ctypes.c_int),
        "hgx_result_count": ([vp, ctypes.c_int], ctypes.c_uint64),
        "hgx_result_copy": ([vp, ctypes.c_int, vp, ctypes.c_size_t], ctypes.c_int),
        "hgx_result_free": ([vp], None),
        "hgx_result_view": ([vp, ctypes.c_int, ctypes.POINTER(vp), u64p], ctypes.c_int),
        "hgx_engine_stage_times": ([vp, ctypes.POINTER(ctypes.c_double), u64p], ctypes.c_int),
        "hgx_engine_expand_stats": ([vp, u64p], ctypes.c_int),
        "hgx_engine_result_stats": ([vp, u64p], ctypes.c_int),
        "hgx_engine_stream": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "hgx_hash_states_noalloc": ([vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32, vp, vp, vp], ctypes.c_int),
        "hgx_estimate_device_bytes": ([ctypes.POINTER(Job), u64p], ctypes.c_int),
        "hgx_device_memory": ([ctypes.c_int, u64p, u64p], ctypes.c_int),
        "hgx_result_views": ([vp, ctypes.POINTER(vp), u64p], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(status: int):
    if status != HGX_OK:
        raise HgxError(status, load_library().hgx_last_error().decode())


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


# ---------------------------------------------------------------------------------------------
# Blob encodings (include/hgx.h)
# ---------------------------------------------------------------------------------------------

def encode_rule(lhs, rhs) -> np.ndarray:
    out = []
    for side in (lhs, rhs):
        out.append(len(side))
        for e in side:
            out.append(len(e))
            out.extend(int(v) for v in e)
    return np.asarray(out, dtype=np.uint32)


def encode_rules(rules) -> np.ndarray:
    parts = [np.asarray([len(rules)], dtype=np.uint32)]
    parts += [encode_rule(lhs, rhs) for lhs, rhs in rules]
    return np.concatenate(parts)


def encode_roots(roots) -> np.ndarray:
    out = [len(roots)]
    for st in roots:
        out.append(len(st))
        for e in st:
            out.append(len(e))
            out.extend(int(v) for v in e)
    return np.asarray(out, dtype=np.uint32)


# ---------------------------------------------------------------------------------------------
# Results
# ---------------------------------------------------------------------------------------------

@dataclass
class EvolveResult:
    """One evolution's result (ids local to the evolution).

    state_hash[s]  WL canonical hash;  state_depth[s];  events[e] = (in, out, rule, step);
    causal[k] = (producer, consumer, edge);  branchial[k] = (a, b);  plus the consumed /
    produced edges per event and (optionally) every state's edge record.
    """

    state_hash: np.ndarray
    state_depth: np.ndarray
    events: np.ndarray
    causal: np.ndarray
    branchial: np.ndarray
    event_cons_off: np.ndarray
    event_cons: np.ndarray
    event_prod: np.ndarray
    state_edge_off: np.ndarray
    state_edge_ids: np.ndarray
    state_arity: np.ndarray
    state_vert_off: np.ndarray
    state_verts: np.ndarray
    num_classes: int
    truncated: bool
    event_signature: np.ndarray = None   # u64 per event (event canonicalisation on), else empty
    num_canonical_events: int = 0        # distinct event signatures (= events when off)

    def canonical_event(self) -> np.ndarray:
        """Per event, the local id of the first event with its signature (itself when event
        canonicalisation is off)."""
        n = len(self.events)
        if self.event_signature is None or len(self.event_signature) != n:
            return np.arange(n, dtype=np.uint32)
        _, first, inv = np.unique(self.event_signature, return_index=True, return_inverse=True)
        return first[inv].astype(np.uint32)

    @property
    def num_states(self) -> int:
        return len(self.state_hash)

    @property
    def num_events(self) -> int:
        return len(self.events)

    def state_edges(self, s: int):
        """Edges (lists of vertex ids) of state s (needs keep_state_edges)."""
        e0, e1 = self.state_edge_off[s], self.state_edge_off[s + 1]
        v = self.state_vert_off[s]
        out = []
        for a in self.state_arity[e0:e1]:
            out.append(self.state_verts[v:v + a].tolist())
            v += a
        return out

    def keys(self) -> dict:
        """The result as schedule-independent sorted key arrays: the distinct WL class hashes,
        the event keys fnv(WL(in), WL(out), rule, step), the causal keys fnv(key(producer),
        key(consumer)) and the branchial keys fnv(min, max) -- the reference's own cross-engine
        normalisation (gpu/tests/test_gpu_vs_cpu_differential.cpp:119-157). Two results are the
        same evolution exactly when these arrays are equal."""
        sh = np.asarray(self.state_hash, dtype=np.uint64)
        ev = np.asarray(self.events, dtype=np.uint32).reshape(-1, 4)
        with np.errstate(over="ignore"):
            def fold(h, x):
                return np.bitwise_xor(h, np.asarray(x, dtype=np.uint64)) * _FNV_PRIME

            ek = np.full(len(ev), _FNV_OFFSET, dtype=np.uint64)
            for col in (sh[ev[:, 0]], sh[ev[:, 1]], ev[:, 2], ev[:, 3]):
                ek = fold(ek, col)
            ca = np.asarray(self.causal, dtype=np.uint32).reshape(-1, 3)
            ck = fold(fold(np.full(len(ca), _FNV_OFFSET, dtype=np.uint64), ek[ca[:, 0]]), ek[ca[:, 1]])
            br = np.asarray(self.branchial, dtype=np.uint32).reshape(-1, 2)
            a, b = ek[br[:, 0]], ek[br[:, 1]]
            bk = fold(fold(np.full(len(br), _FNV_OFFSET, dtype=np.uint64), np.minimum(a, b)),
                      np.maximum(a, b))
        return {"state_hashes": np.unique(sh), "event_keys": np.sort(ek),
                "causal_keys": np.sort(ck), "branchial_keys": np.sort(bk)}

    def same_as(self, other: "EvolveResult") -> bool:
        """Exact equality of the two results' key multisets (see keys())."""
        a, b = self.keys(), other.keys()
        return all(np.array_equal(a[k], b[k]) for k in a)

    def bytes(self) -> int:
        return sum(getattr(self, f).nbytes for f in (
            "state_hash", "state_depth", "events", "causal", "branchial", "event_cons_off",
            "event_cons", "event_prod", "state_edge_off", "state_edge_ids", "state_arity",
            "state_vert_off", "state_verts"))


class _ResultOwner:
    """Frees an hgx_result once no numpy view of its memory is left."""

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        try:
            load_library().hgx_result_free(self.handle)
        except Exception:
            pass


_ARR_TYPES = {ARR_STATE_HASH: np.uint64, ARR_EVENT_SIG: np.uint64, ARR_STATE_ARITY: np.uint8}
_ARR_SHAPES = {ARR_EVENTS: 4, ARR_CAUSAL: 3, ARR_BRANCHIAL: 2, ARR_EVENT_PROD: 2}


def _read_result(handle) -> EvolveResult:
    """Zero-copy: every array is a numpy view of the result's host memory (page-locked for a
    single-evolution result); the handle is freed when the last view is released."""
    L = load_library()
    owner = _ResultOwner(handle)
    cnt = lambda w: int(L.hgx_result_count(handle, w))  # noqa: E731
    arrays = {}
    ptrs = (ctypes.c_void_p * 14)()
    counts = (ctypes.c_uint64 * 14)()
    _check(L.hgx_result_views(handle, ptrs, counts))
    for what in range(14):
        dt = _ARR_TYPES.get(what, np.uint32)
        n, p = int(counts[what]), ptrs[what]
        if n == 0 or not p:
            a = np.zeros(0, dt)
        else:
            buf = (ctypes.c_char * (n * np.dtype(dt).itemsize)).from_address(p)
            buf._owner = owner
            a = np.frombuffer(buf, dtype=dt)
        w = _ARR_SHAPES.get(what)
        arrays[what] = a.reshape(-1, w) if w else a
    return EvolveResult(
        state_hash=arrays[ARR_STATE_HASH], state_depth=arrays[ARR_STATE_DEPTH],
        events=arrays[ARR_EVENTS], causal=arrays[ARR_CAUSAL], branchial=arrays[ARR_BRANCHIAL],
        event_cons_off=arrays[ARR_EVENT_CONS_OFF], event_cons=arrays[ARR_EVENT_CONS],
        event_prod=arrays[ARR_EVENT_PROD], state_edge_off=arrays[ARR_STATE_EDGE_OFF],
        state_edge_ids=arrays[ARR_STATE_EDGE_IDS], state_arity=arrays[ARR_STATE_ARITY],
        state_vert_off=arrays[ARR_STATE_VERT_OFF], state_verts=arrays[ARR_STATE_VERTS],
        num_classes=cnt(COUNT_CLASSES), truncated=bool(cnt(COUNT_TRUNCATED)),
        event_signature=arrays[ARR_EVENT_SIG], num_canonical_events=cnt(COUNT_CANONICAL_EVENTS))


def estimate_device_bytes(evolution) -> int:
    """Estimated device bytes of one evolution (rules, roots, steps, cap) -- the engine's own
    estimate through the C-ABI (hgx_estimate_device_bytes); needs no device."""
    jobs, _keep = Engine.make_jobs([evolution])
    b = ctypes.c_uint64()
    _check(load_library().hgx_estimate_device_bytes(ctypes.byref(jobs[0]), ctypes.byref(b)))
    return int(b.value)


class Engine:
    """A device engine (one CUDA stream and its device arrays). Reusable across calls."""

    def __init__(self, device: int = 0, keep_state_edges: bool = True, causal: bool = True,
                 branchial: bool = True, timing: bool = False):
        L = load_library()
        h = ctypes.c_void_p()
        _check(L.hgx_engine_create(int(device), ctypes.byref(h)))
        self._h = h
        self._L = L
        self.set_option(OPT_KEEP_STATE_EDGES, keep_state_edges)
        self.set_option(OPT_RECORD_CAUSAL, causal)
        self.set_option(OPT_RECORD_BRANCHIAL, branchial)
        self.set_option(OPT_TIMING, timing)

    def close(self):
        if getattr(self, "_h", None):
            self._L.hgx_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, opt: int, value) -> None:
        _check(self._L.hgx_engine_set_option(self._h, int(opt), int(value)))

    def evolve(self, rules, roots, steps, quotient=True, max_states=0) -> EvolveResult:
        L = self._L
        _check(L.hgx_engine_clear_rules(self._h))
        for lhs, rhs in rules:
            b = encode_rule(lhs, rhs)
            _check(L.hgx_engine_add_rule(self._h, _u32p(b), len(b)))
        self.set_option(OPT_QUOTIENT, quotient)
        self.set_option(OPT_MAX_STATES, max_states)
        rb = encode_roots(roots)
        out = ctypes.c_void_p()
        _check(L.hgx_evolve(self._h, _u32p(rb), len(rb), int(steps), ctypes.byref(out)))
        return _read_result(out.value)

    @staticmethod
    def make_jobs(evolutions):
        """ctypes job array for a list of workloads.Evolution (keeps the blobs alive)."""
        blobs = []
        jobs = (Job * len(evolutions))()
        for i, ev in enumerate(evolutions):
            rb, sb = encode_rules(ev.rules), encode_roots(ev.roots)
            blobs += [rb, sb]
            jobs[i] = Job(_u32p(rb), len(rb), _u32p(sb), len(sb), int(ev.steps), int(bool(ev.quotient)),
                          int(ev.max_states))
        return jobs, blobs

    def evolve_batch(self, evolutions, jobs=None):
        if jobs is None:
            jobs, _keep = self.make_jobs(evolutions)
        n = len(jobs)
        outs = (ctypes.c_void_p * n)()
        _check(self._L.hgx_evolve_batch(self._h, jobs, n, outs))
        return [_read_result(outs[i]) for i in range(n)]

    # --- serving ---
    def serve_reset(self):
        _check(self._L.hgx_serve_reset(self._h))

    def serve_admit(self, job: Job) -> int:
        i = ctypes.c_uint32()
        _check(self._L.hgx_serve_admit(self._h, ctypes.byref(job), ctypes.byref(i)))
        return int(i.value)

    def serve_admit_batch(self, jobs, n: int | None = None) -> list:
        """Admit the first n jobs of a Job array in one call; returns their evolution ids."""
        n = len(jobs) if n is None else n
        ids = (ctypes.c_uint32 * max(n, 1))()
        _check(self._L.hgx_serve_admit_batch(self._h, jobs, n, ids))
        return list(ids[:n])

    def serve_step(self) -> bool:
        a = ctypes.c_int()
        _check(self._L.hgx_serve_step(self._h, ctypes.byref(a)))
        return bool(a.value)

    def serve_take_finished(self, cap: int = 1 << 16):
        ids = (ctypes.c_uint32 * cap)()
        n = ctypes.c_uint32()
        _check(self._L.hgx_serve_take_finished(self._h, ids, cap, ctypes.byref(n)))
        return list(ids[: n.value])

    def serve_collect(self, evo: int) -> EvolveResult:
        out = ctypes.c_void_p()
        _check(self._L.hgx_serve_collect(self._h, int(evo), ctypes.byref(out)))
        return _read_result(out.value)

    def serve_collect_batch(self, evos) -> list:
        """Collect several finished evolutions with one device finalisation and one copy."""
        n = len(evos)
        if n == 0:
            return []
        ids = (ctypes.c_uint32 * n)(*[int(e) for e in evos])
        outs = (ctypes.c_void_p * n)()
        _check(self._L.hgx_serve_collect_batch(self._h, ids, n, outs))
        return [_read_result(outs[i]) for i in range(n)]

    def device_bytes(self) -> int:
        b = ctypes.c_uint64()
        _check(self._L.hgx_serve_device_bytes(self._h, ctypes.byref(b)))
        return int(b.value)

    def expand_stats(self):
        out = (ctypes.c_uint64 * 11)()
        _check(self._L.hgx_engine_expand_stats(self._h, out))
        return dict(zip(("stage_bytes", "hbm_bytes", "children", "wl_rounds", "launches",
                         "warp_stage_bytes", "warp_hbm_bytes", "warp_children", "warp_rounds",
                         "warp_ns", "walk_launches"), list(out)))

    def result_stats(self):
        """Whether the last result was streamed (copied out range by range during the run) and
        in how many chunks."""
        out = (ctypes.c_uint64 * 2)()
        _check(self._L.hgx_engine_result_stats(self._h, out))
        return {"streamed": bool(out[0]), "chunks": int(out[1])}

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(self._L.hgx_engine_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def counts(self, rules, roots, steps, quotient=True, max_states=0):
        """Evolve with the result left on the device; returns the counts only."""
        self.set_option(OPT_READBACK, 0)
        try:
            L = self._L
            _check(L.hgx_engine_clear_rules(self._h))
            for lhs, rhs in rules:
                b = encode_rule(lhs, rhs)
                _check(L.hgx_engine_add_rule(self._h, _u32p(b), len(b)))
            self.set_option(OPT_QUOTIENT, quotient)
            self.set_option(OPT_MAX_STATES, max_states)
            rb = encode_roots(roots)
            out = ctypes.c_void_p()
            _check(L.hgx_evolve(self._h, _u32p(rb), len(rb), int(steps), ctypes.byref(out)))
            try:
                cnt = lambda w: int(L.hgx_result_count(out, w))  # noqa: E731
                return {"states": cnt(COUNT_STATES), "events": cnt(COUNT_EVENTS),
                        "classes": cnt(COUNT_CLASSES), "causal": cnt(COUNT_CAUSAL),
                        "branchial": cnt(COUNT_BRANCHIAL), "truncated": bool(cnt(COUNT_TRUNCATED)),
                        "canonical_events": cnt(COUNT_CANONICAL_EVENTS)}
            finally:
                L.hgx_result_free(out)
        finally:
            self.set_option(OPT_READBACK, 1)

    def stage_times(self):
        out = (ctypes.c_double * 8)()
        launches = ctypes.c_uint64()
        _check(self._L.hgx_engine_stage_times(self._h, out, ctypes.byref(launches)))
        names = ("count", "scan", "expand", "select", "materialize", "branchial", "roots", "total")
        return dict(zip(names, list(out))), int(launches.value)


# ---------------------------------------------------------------------------------------------
# Reference-shaped API
# ---------------------------------------------------------------------------------------------

MAX_PATTERN_EDGES, MAX_ARITY, MAX_VARS = 16, 16, 32


@dataclass
class RewriteRule:
    """A rule: LHS / RHS pattern edges over variables (pattern.hpp:71-140)."""

    index: int
    lhs: list
    rhs: list

    @property
    def num_lhs_edges(self):
        return len(self.lhs)

    @property
    def num_rhs_edges(self):
        return len(self.rhs)

    def new_var_mask(self) -> int:
        lm = 0
        rm = 0
        for e in self.lhs:
            for v in e:
                lm |= 1 << v
        for e in self.rhs:
            for v in e:
                rm |= 1 << v
        return rm & ~lm


class RuleBuilder:
    """Fluent builder (pattern.hpp:142-206); raises ValueError where the reference throws
    std::length_error (more than 16 edges, arity above 16, variable index >= 32)."""

    def __init__(self, index: int = 0):
        self._rule = RewriteRule(index, [], [])

    def _edge(self, side, vars_):
        vars_ = [int(v) for v in vars_]
        if len(side) >= MAX_PATTERN_EDGES:
            raise ValueError("RuleBuilder: exceeds MAX_PATTERN_EDGES")
        if len(vars_) > MAX_ARITY:
            raise ValueError("RuleBuilder: edge arity exceeds MAX_ARITY")
        if any(v < 0 or v >= MAX_VARS for v in vars_):
            raise ValueError("RuleBuilder: pattern variable index exceeds MAX_VARS")
        side.append(vars_)
        return self

    def lhs(self, vars_):
        return self._edge(self._rule.lhs, vars_)

    def rhs(self, vars_):
        return self._edge(self._rule.rhs, vars_)

    def build(self) -> RewriteRule:
        return RewriteRule(self._rule.index, [list(e) for e in self._rule.lhs],
                           [list(e) for e in self._rule.rhs])


def make_rule(index: int = 0) -> RuleBuilder:
    return RuleBuilder(index)


class CausalGraph:
    def __init__(self, res: EvolveResult | None):
        self._r = res

    def get_causal_edges(self):
        """(producer, consumer, edge) triples."""
        return [] if self._r is None else [tuple(map(int, t)) for t in self._r.causal]

    def get_branchial_edges(self):
        """(event1, event2) pairs with event1 < event2."""
        return [] if self._r is None else [tuple(map(int, t)) for t in self._r.branchial]

    def num_causal_edges(self):
        return 0 if self._r is None else len(self._r.causal)

    def num_branchial_edges(self):
        return 0 if self._r is None else len(self._r.branchial)


class Hypergraph:
    """Holds the evolution a ParallelEvolutionEngine produced (hypergraph.hpp:567-811)."""

    def __init__(self):
        self.result: EvolveResult | None = None
        self._event_keys = EVENT_SIG_NONE

    def set_event_signature_keys(self, keys: int):
        """Event canonicalisation (hypergraph.hpp:778): hgcommon EventSignatureKeys bits over the
        WL hashes (1 input, 2 output, 4 step, 8 rule); read by the engine at evolve()."""
        if int(keys) & ~0xF:
            raise ValueError("edge-rank event keys need an exact canonical labelling (not provided)")
        self._event_keys = int(keys)

    def event_signature_keys(self) -> int:
        return self._event_keys

    def num_raw_events(self) -> int:
        return 0 if self.result is None else self.result.num_events

    def num_states(self) -> int:
        """Raw states: every root plus one per event (hypergraph.hpp:567)."""
        if self.result is None:
            return 0
        roots = int(np.sum(self.result.state_depth == 0))
        return roots + self.result.num_events

    def num_canonical_states(self) -> int:
        """Distinct WL canonical hashes."""
        return 0 if self.result is None else int(self.result.num_classes)

    def num_events(self) -> int:
        """Canonical events when event canonicalisation is on (hypergraph.cpp:1639-1644)."""
        if self.result is None:
            return 0
        return int(self.result.num_canonical_events) if self._event_keys else self.result.num_events

    def get_canonical_event(self, eid: int) -> int:
        return int(self.result.canonical_event()[eid])

    def get_or_compute_canonical_hash(self, sid: int) -> int:
        return int(self.result.state_hash[sid])

    def causal_graph(self) -> CausalGraph:
        return CausalGraph(self.result)


class ParallelEvolutionEngine:
    """Same call sequence as the reference engine (parallel_evolution.hpp:743-1041); the
    evolution runs on the GPU. num_threads is accepted for signature compatibility."""

    def __init__(self, hg: Hypergraph, num_threads: int = 0, device: int = 0):
        self._hg = hg
        self._rules: list[RewriteRule] = []
        self._quotient = False
        self._max_states = 0
        self._engine = Engine(device)

    def add_rule(self, rule: RewriteRule):
        self._rules.append(rule)

    def set_explore_from_canonical_states_only(self, enable: bool):
        self._quotient = bool(enable)

    def set_transitive_reduction(self, enable: bool):
        self._engine.set_option(OPT_TRANSITIVE_REDUCTION, bool(enable))

    def set_max_states(self, n: int):
        self._max_states = int(n)

    def num_states(self):
        return self._hg.num_states()

    def num_events(self):
        return self._hg.num_events()

    def num_canonical_states(self):
        return self._hg.num_canonical_states()

    def evolve(self, initial, steps: int):
        """initial: a list of edges (one root) or a list of states (several roots)."""
        if not self._rules:
            return
        roots = initial if initial and isinstance(initial[0][0], (list, tuple)) else [initial]
        rules = [(r.lhs, r.rhs) for r in sorted(self._rules, key=lambda r: r.index)]
        self._engine.set_option(OPT_EVENT_SIGNATURE_KEYS, self._hg.event_signature_keys())
        self._hg.result = self._engine.evolve(rules, roots, steps, self._quotient, self._max_states)
