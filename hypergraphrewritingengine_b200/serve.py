"""Continuous-batching request loop for evolve requests.

The reference serves requests strictly one at a time (paclet_source/hg_evolve_main.cpp:99-246,
``run_serve``: read a frame, run it to completion on a process-static evolver, reply). Here a
request is admitted into the running engine as soon as it has arrived and its estimated device
footprint fits the memory budget; every loop iteration advances ALL admitted requests by one
level in shared launches (each at its own depth: requests admitted at different times are at
different levels of their evolutions); a request that has finished is collected -- its result
copied to the host -- while the others keep running, and the engine's memory is reclaimed
whenever it goes idle.

``Server.run`` returns one ``Record`` per request with its arrival, admission and completion
times and its result; ``serve_plain`` is the same stream served one request per call (the plain
path), for comparison.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import api


@dataclass
class Record:
    rid: int
    arrival: float
    admitted: float = -1.0
    finished: float = -1.0
    result: object = None
    meta: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def estimate_bytes(ev) -> int:
    """Device-memory estimate of one evolve request: the engine's own estimate (states, events,
    relations and dedup tables from the rules, roots, step budget and state cap; an uncapped
    request is estimated at the states its step budget can reach, at most 2^22), through the
    C-ABI (hgx_estimate_device_bytes; reference: hg_gpu::estimated_device_bytes)."""
    return api.estimate_device_bytes(ev)


class Server:
    """Continuous batching over one api.Engine."""

    def __init__(self, engine: api.Engine, memory_budget: float = 140e9, max_active: int = 1 << 16,
                 track_device_bytes: bool = False):
        self.eng = engine
        self.budget = memory_budget
        self.max_active = max_active
        # admission bookkeeping of the last run: requests admitted per admission call, the
        # largest estimated footprint admitted at once, and (when tracked) the largest device
        # footprint the engine reported after a step
        self.track = track_device_bytes
        self.admit_sizes: list[int] = []
        self.peak_reserved = 0
        self.peak_device_bytes = 0

    def run(self, arrivals, realtime: bool = True, admit_per_step: int | None = None):
        """Serve a stream. arrivals: list of (arrival_time_s, workloads.Evolution), sorted by
        time. realtime=False admits `admit_per_step` requests before every step instead of
        following the clock (deterministic staggering, used by the tests)."""
        if admit_per_step is not None and admit_per_step < 1:
            raise ValueError(f"admit_per_step must be >= 1 (got {admit_per_step}): "
                             "nothing would ever be admitted")
        eng = self.eng
        eng.serve_reset()
        self.admit_sizes, self.peak_reserved, self.peak_device_bytes = [], 0, 0
        recs = [Record(i, t) for i, (t, _) in enumerate(arrivals)]
        pending = collections.deque(range(len(arrivals)))
        active = {}            # engine evolution id -> request index
        reserved = 0           # estimated bytes of the admitted requests
        keep = {}              # job arrays of the admitted requests
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        def collect_finished():
            nonlocal reserved
            done = eng.serve_take_finished()
            if not done:
                return
            results = eng.serve_collect_batch(done)   # one finalisation for all of them
            t_done = now()
            for evo, res in zip(done, results):
                i = active.pop(evo)
                recs[i].result = res
                recs[i].finished = t_done
                reserved -= recs[i].meta.pop("est")
                keep.pop(i, None)

        while pending or active:
            # admission: arrived requests that fit the memory budget, admitted in one call
            take = []
            while pending and len(active) + len(take) < self.max_active:
                i = pending[0]
                t_arr, ev = arrivals[i]
                if realtime and t_arr > now():
                    break
                if not realtime and admit_per_step is not None and len(take) >= admit_per_step:
                    break
                est = estimate_bytes(ev)
                if (active or take) and reserved + est > self.budget:
                    break
                pending.popleft()
                take.append(i)
                recs[i].meta["est"] = est
                reserved += est
            if take:
                self.admit_sizes.append(len(take))
                self.peak_reserved = max(self.peak_reserved, reserved)
                jobs, blobs = api.Engine.make_jobs([arrivals[i][1] for i in take])
                ids = eng.serve_admit_batch(jobs, len(take))
                t_adm = now()
                for i, evo in zip(take, ids):
                    active[evo] = i
                    recs[i].admitted = t_adm
                    keep[i] = (jobs, blobs)
            collect_finished()                 # zero-step requests finish at admission
            if not active:
                if not pending:
                    break
                eng.serve_reset()              # idle: reclaim the engine's memory
                if realtime:
                    wait = arrivals[pending[0]][0] - now()
                    if wait > 0:
                        time.sleep(wait)
                continue
            eng.serve_step()
            if self.track:
                self.peak_device_bytes = max(self.peak_device_bytes, eng.device_bytes())
            collect_finished()
        return recs


def serve_plain(engine: api.Engine, arrivals, realtime: bool = True):
    """The same stream, one request per call in arrival order (the plain path)."""
    recs = [Record(i, t) for i, (t, _) in enumerate(arrivals)]
    t0 = time.perf_counter()
    for i, (t_arr, ev) in enumerate(arrivals):
        if realtime:
            wait = t_arr - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        recs[i].admitted = time.perf_counter() - t0
        recs[i].result = engine.evolve(ev.rules, ev.roots, ev.steps, quotient=ev.quotient,
                                       max_states=ev.max_states)
        recs[i].finished = time.perf_counter() - t0
    return recs


def summarize(recs):
    lat = np.array([r.latency for r in recs]) * 1e3
    span = max(r.finished for r in recs) - min(r.arrival for r in recs)
    events = sum(r.result.num_events for r in recs)
    states = sum(r.result.num_states for r in recs)
    return {"requests": len(recs), "events": int(events), "unique_states": int(states),
            "makespan_ms": span * 1e3, "events_per_s": events / span,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}
