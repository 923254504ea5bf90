#!/usr/bin/env python
"""Benchmark of the multiway evolution step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A "step" is one complete WL-quotient evolution of the single large workload: rule
{{x,y},{x,z}} -> {{x,z},{x,w},{y,w},{z,w}} (w fresh) from {{1,1},{1,1}}, 8 levels, WL dedup, capped
at 2,000,000 unique states, causal + branchial relations recorded.  Inputs are synthetic (the
rule and the initial state), generated in-process.

* value   events/s over all ranks, device-resident (the result stays in HBM; counts read back),
          timed with CUDA events on the engine's stream, L2 flushed (256 MB write) before each step.
* e2e     the same metric through the C-ABI call a user makes (hgx_evolve with host buffers):
          rule/state blobs copied in and the whole result (states, events, causal, branchial)
          copied out every step, timed on the host clock around the call.
* roofline  the dominant kernel (k_expand: join + rewrite + WL hash + dedup insert, fused), its
          algorithmic bytes per launch over its CUDA-event launch time, against the measured HBM
          copy bandwidth (MEASURED_PEAKS.json).
* cpu_baseline  the reference CPU engine (oracle/_ref/hgref, compiled from the reference's own
          sources) on a bounded sample of the same workload in WL mode (every state WL-hashed):
          C2's rule and initial state unfolded to 4 levels, all host threads. The reference has no
          WL-keyed quotient exploration.
* c1      the one workload both engines run identically (C1: triangle, 5 steps, full multiway):
          this path's device-resident and end-to-end rates beside the reference engine's over a
          thread sweep (1 thread and the best), and the ratios.
* c3      C3 (ternary, 6 levels, WL quotient) with incremental match forwarding off and on,
          results compared exactly (key multisets).
* batched  1024 random evolutions (seeded generator) in one batched pipeline vs. the plain path
          (one evolution per call), same GPU, identical per-evolution outputs (key multisets).
* served  a Poisson request stream served with continuous batching vs. one request per call.

Multi-GPU: the single large evolution does not shard; --gpus N runs N replicas of it under
torchrun and reports the aggregate with the max-over-ranks time ("scaling": "weak"). The batched
workload does shard (independent evolutions, no exchange step): the line adds "sharded_batch",
1024 random evolutions per rank split by shard.assign, max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "events/s (WL-quotient multiway evolution; unique states/s alongside)"
WORKLOAD = ("c2: {{x,y},{x,z}}->{{x,z},{x,w},{y,w},{z,w}} from {{1,1},{1,1}}, 8 steps, WL dedup, "
            "cap 2,000,000 unique states, causal+branchial recorded")
C1_WORKLOAD = ("c1: {{x,y},{y,z}}->{{x,y},{y,z},{z,x}} from the triangle {{1,2},{2,3},{3,1}}, "
               "5 steps, full multiway, WL mode, causal+branchial recorded")
C3_WORKLOAD = ("c3: {{x,y,z},{z,u,v}}->{{w,w,y},{w,x,u},{v,u,z},{y,v,w}} from {{1,1,1},{1,1,1}}, "
               "6 steps, WL quotient, causal+branchial recorded")


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled while running: through NVML every
    10 ms on the device torch uses (found by PCI bus id), else nvidia-smi every 200 ms. Reads
    only; changes no setting."""

    # NVML clock-event reason bits (nvmlClocksEventReason*)
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.lines = []
        self.samples = []          # (sm MHz, max MHz, reason bits) from NVML
        self.proc = None
        self.stop = threading.Event()
        self.t = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.gpu)
        bus = getattr(props, "pci_bus_id", None)
        if bus is None:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
        dom, dev = getattr(props, "pci_domain_id", 0), getattr(props, "pci_device_id", 0)
        for i in range(pynvml.nvmlDeviceGetCount()):
            h = pynvml.nvmlDeviceGetHandleByIndex(i)
            pci = pynvml.nvmlDeviceGetPciInfo(h)
            if (pci.bus, pci.device, pci.domain) == (bus, dev, dom):
                return pynvml, h
        raise RuntimeError("no NVML device with the PCI address torch reports")

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def run():
                while not self.stop.is_set():
                    try:
                        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                             nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
                    except Exception:
                        pass
                    self.stop.wait(0.01)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
            self.source = "nvml, 10 ms"
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.source = "nvidia-smi, 200 ms"
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        elif self.t is not None:
            self.t.join(timeout=1)

    def summary(self):
        mhz, mx, reasons = [], 0.0, set()
        for sm, smax, bits in self.samples:
            mhz.append(float(sm))
            mx = max(mx, float(smax))
            reasons.update(n for b, n in self.REASONS.items() if bits & b)
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(mhz), "source": self.source}


def max_over_ranks(dist, value: float, device: str = "cuda") -> float:
    """Max of a per-rank time over all ranks (a collective every rank must call)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def profile_traffic():
    """dram bytes per lane-expand launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "k_expand.c2-8step.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_per_launch_bytes"):
            return float(line.split("=")[1].split()[0])
    return None


def _thread_counts():
    """1, 2, 4, ... below the host's thread count, then the thread count itself."""
    n = os.cpu_count() or 1
    out, t = [], 1
    while t < n:
        out.append(t)
        t *= 2
    return out + [n]


def cpu_baseline_reference(threads: int | None = None, levels: int = 4, reps: int = 3):
    """Reference CPU engine on a bounded sample of the C2 workload, in WL mode: its
    StateCanonicalizationMode::None, where every state reports the WL hash computed as it is
    created (hypergraph/src/hypergraph.cpp:180-197), i.e. the same per-event work as this path
    (join, rewrite, WL hash, causal and branchial edges). The reference has no WL-keyed quotient
    exploration, so the sample is C2's rule and initial state unfolded in full to `levels` levels
    (4: 9,938 events; 5 levels exceed 48 GB of host memory in the reference)."""
    from hypergraphrewritingengine_b200 import workloads as W
    from oracle import pyoracle
    ev = W.config2(levels)
    threads = threads or os.cpu_count() or 1
    if os.path.exists(pyoracle.REF_BIN):
        best = None
        for _ in range(reps):
            r = pyoracle.run_reference(ev.rules, ev.roots, ev.steps, quotient=False, threads=threads,
                                       timeout=600)
            best = r if best is None or r["ms"] < best["ms"] else best
        r = best
        return {"value": r["events"] / (r["ms"] / 1e3), "unit": "events/s", "cores": threads,
                "kind": "reference",
                "sample": f"reference engine (oracle/_ref, built from its own sources) in WL mode "
                          f"(None canonicalisation: every state WL-hashed) on C2's rule and initial "
                          f"state unfolded to {levels} levels: {r['events']} events, "
                          f"{r['wl_classes']} WL classes, {r['causal']} causal, {r['branchial']} "
                          f"branchial in {r['ms']:.1f} ms (best of {reps})"}
    t = time.perf_counter()
    r = pyoracle.evolve(ev.rules, ev.roots, 7, quotient=True)
    dt = time.perf_counter() - t
    return {"value": len(r["events"]) / dt, "unit": "events/s", "cores": 1, "kind": "port",
            "sample": f"oracle restatement, WL quotient to 7 levels: {len(r['events'])} events in {dt:.1f} s"}


def reference_c1_sweep():
    """C1 exactly as configured (triangle, 5 steps, full multiway, WL mode, causal + branchial)
    on the reference CPU engine, over a thread sweep: the one workload both engines run
    identically."""
    from hypergraphrewritingengine_b200 import workloads as W
    from oracle import pyoracle
    if not os.path.exists(pyoracle.REF_BIN):
        return None
    ev = W.config1()
    runs = []
    for th in _thread_counts():
        r = pyoracle.run_reference(ev.rules, ev.roots, ev.steps, quotient=False, threads=th,
                                   timeout=900)
        runs.append({"threads": th, "ms": r["ms"], "events": r["events"],
                     "events_per_s": r["events"] / (r["ms"] / 1e3)})
    best = min(runs, key=lambda x: x["ms"])
    one = runs[0]
    return {"workload": C1_WORKLOAD, "kind": "reference", "events": best["events"],
            "sweep": runs, "best": {"threads": best["threads"], "ms": best["ms"],
                                    "events_per_s": best["events_per_s"]},
            "one_thread": {"ms": one["ms"], "events_per_s": one["events_per_s"]}}


def run_reference_arm(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline_reference(cores, reps=1)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.mean(vals)
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "events/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD + " (reference: bounded sample, WL mode, C2's rule "
                                              "and initial state unfolded to 4 levels)"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    c1 = reference_c1_sweep()
    if c1:
        line["c1"] = c1
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the batched comparison")
    ap.add_argument("--levels", type=int, default=8)
    ap.add_argument("--lane-join", type=int, default=0, choices=[0, 1, 2],
                    help="small-state join: 0 autotuned (default), 1 warp join, 2 lane walk")
    ap.add_argument("--profile-run", action="store_true",
                    help="run the workload once, device-resident, and exit (for profilers)")
    ap.add_argument("--profile-workload", default="c2", choices=["c2", "c4", "large"],
                    help="--profile-run workload: c2 (--levels levels), c4 (1024 random "
                         "evolutions) or large (256 random evolutions with 65-256-edge states)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile_run:
        from hypergraphrewritingengine_b200 import Engine
        from hypergraphrewritingengine_b200 import workloads as W
        from hypergraphrewritingengine_b200 import api
        eng = Engine(0)
        eng.set_option(api.OPT_LANE_JOIN, args.lane_join)
        if args.profile_workload == "c2":
            ev = W.config2(args.levels)
            c = eng.counts(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        else:
            evs = (W.config4(n=1024) if args.profile_workload == "c4" else
                   [W.random_evolution(i, seed=0x1A26E, edges_lo=65, edges_hi=256, steps_lo=2,
                                       steps_hi=4) for i in range(256)])
            jobs, keep = eng.make_jobs(evs)
            out = (api.ctypes.c_void_p * len(evs))()
            eng.set_option(api.OPT_READBACK, 0)
            api._check(eng._L.hgx_evolve_batch(eng._h, jobs, len(evs), out))
            c = {"events": sum(int(eng._L.hgx_result_count(out[i], 1)) for i in range(len(evs)))}
            for i in range(len(evs)):
                eng._L.hgx_result_free(out[i])
        print(json.dumps(c))
        return

    import numpy as np
    import torch

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from hypergraphrewritingengine_b200 import Engine, encode_roots, encode_rules
    from hypergraphrewritingengine_b200 import workloads as W

    ev = W.config2(args.levels)
    eng = Engine(local)
    from hypergraphrewritingengine_b200 import api as _api
    eng.set_option(_api.OPT_LANE_JOIN, args.lane_join)
    stream = torch.cuda.ExternalStream(eng.stream(), device=torch.device("cuda", local))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")   # 256 MB > 126 MB L2

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        counts = eng.counts(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)

    # ---- timed region (device-resident); the expand kernel launches are timed with event pairs on
    # the engine stream (no syncs); the other stages are timed on one extra step afterwards
    from hypergraphrewritingengine_b200 import api
    eng.set_option(api.OPT_TIMING, 2)
    expand_ms = 0.0
    expand_launches = walk_launches = 0
    stage_bytes = hbm_bytes = children = rounds = 0
    launches = 0
    step_ms = []
    with ClockSampler(local) as clocks:
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            counts = eng.counts(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            st, nl = eng.stage_times()
            xs = eng.expand_stats()
            expand_ms += st["expand"]
            expand_launches += xs["launches"]
            walk_launches += xs["walk_launches"]
            stage_bytes += xs["stage_bytes"]
            hbm_bytes += xs["hbm_bytes"]
            children += xs["children"]
            rounds += xs["wl_rounds"]
            launches += nl
        barrier()
    eng.set_option(api.OPT_TIMING, 1)
    eng.counts(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
    st_all, _ = eng.stage_times()
    eng.set_option(api.OPT_TIMING, 0)
    t_ms = max_over_ranks(dist, sum(step_ms) / len(step_ms))
    events = counts["events"]
    states = counts["states"]
    value = world * events / (t_ms / 1e3)

    # ---- e2e through the C-ABI with host buffers; the result is what the reference's
    # hg_gpu::evolve returns by default (edge_identity false: state edge contents without their
    # global edge ids)
    eng.set_option(_api.OPT_KEEP_STATE_EDGE_IDS, 0)
    rb, sb = encode_rules(ev.rules), encode_roots(ev.roots)
    h2d = rb.nbytes + sb.nbytes
    e2e_s = []
    d2h = 0
    # four untimed calls first: the first result is copied whole and sizes the page-locked blocks
    # the later ones stream into; a result stays alive while the next call runs, so those blocks
    # are allocated twice before they start being recycled
    n_untimed = 4
    streamed = []
    for i in range(n_untimed + args.steps):
        barrier()
        t0 = time.perf_counter()
        res = eng.evolve(ev.rules, ev.roots, ev.steps, quotient=True, max_states=ev.max_states)
        dt = time.perf_counter() - t0
        if i >= n_untimed:
            e2e_s.append(dt)
            streamed.append(eng.result_stats()["streamed"])
        d2h = res.bytes()
        assert res.num_events == events and res.num_states == states
    e2e_t = max_over_ranks(dist, statistics.mean(e2e_s))
    eng.set_option(_api.OPT_KEEP_STATE_EDGE_IDS, 1)
    sharded = sharded_batch(eng, dist, world, rank, barrier) if world > 1 and not args.no_extras else None

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peak, peak_kind = peaks()
    per_launch_bytes = stage_bytes / max(expand_launches, 1)
    per_launch_s = expand_ms / 1e3 / max(expand_launches, 1)
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else None
    traffic = profile_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded rule and initial state; no dataset)",
        "config": {"workload": WORKLOAD, "levels": args.levels, "parallelism": f"replicas x{world}",
                   "l2": "flushed before every step (256 MB device write)",
                   "events_per_step": events, "unique_states_per_step": states,
                   "classes": counts["classes"], "causal_per_step": counts["causal"],
                   "branchial_per_step": counts["branchial"], "truncated_at_cap": counts["truncated"]},
        "unique_states_per_s": world * states / (t_ms / 1e3),
        "e2e": {"value": world * events / e2e_t, "unit": "events/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_t * 1e3,
                "result": "every state (WL hash, depth, edge arities and vertices), every event "
                          "(in, out, rule, step, consumed and produced edges), causal triples, "
                          "branchial pairs; state edge ids left out as in hg_gpu::EvolveResult "
                          "by default (EvolveInput::edge_identity false)",
                "streamed_calls": int(sum(streamed)), "untimed_calls": n_untimed,
                "copy": "each finished frontier range's share of the result copied to page-locked "
                        "host memory on a second stream while the later ranges compute "
                        "(HGX_OPT_STREAM_RESULT)"},
        "roofline": {"bound": "hbm", "kernel": "k_expand_lanes2 (lane expand)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (copy bandwidth)",
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "fused_hbm_bytes_per_launch": hbm_bytes / max(expand_launches, 1),
                     "launch_ms": per_launch_s * 1e3, "launches": expand_launches,
                     "lane_join": {"walk_launches": walk_launches,
                                   "warp_join_launches": expand_launches - walk_launches},
                     "children_hashed": children, "wl_rounds": rounds,
                     "stage_ms_extra_step": {k: round(v, 3) for k, v in st_all.items()}},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if sharded:
        line["sharded_batch"] = sharded
    if world == 1:
        line["cpu_baseline"] = cpu_baseline_reference()
        if not args.no_extras:
            line["c1"] = c1_vs_reference(eng, stream, flush)
            line["c3"] = c3_forwarding(eng, stream, flush)
            line["batched"] = batched_vs_plain(eng)
            line["batched_cap_65536"] = batched_vs_plain(eng, max_states=1 << 16)
            line["join_index"] = join_index_ab(eng)
            line["served"] = served_vs_plain(eng)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _device_ms(eng, stream, flush, ev, reps):
    """Mean CUDA-event time of one device-resident evolution (L2 flushed before each)."""
    import torch
    for _ in range(2):
        c = eng.counts(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
    ms = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c = eng.counts(ev.rules, ev.roots, ev.steps, quotient=ev.quotient, max_states=ev.max_states)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.mean(ms), c


def c1_vs_reference(eng, stream, flush, reps=20):
    """C1 exactly as configured on both engines: this path (device-resident and end to end
    through the C-ABI) against the reference CPU engine's thread sweep."""
    from hypergraphrewritingengine_b200 import workloads as W
    ev = W.config1()
    dev_ms, c = _device_ms(eng, stream, flush, ev, reps)
    e2e = []
    for i in range(2 + reps):
        t0 = time.perf_counter()
        res = eng.evolve(ev.rules, ev.roots, ev.steps, quotient=False)
        if i >= 2:
            e2e.append(time.perf_counter() - t0)
    e2e_ms = statistics.mean(e2e) * 1e3
    out = {"workload": C1_WORKLOAD, "events": c["events"], "raw_states": c["states"],
           "wl_classes": len(set(res.state_hash.tolist())), "causal": c["causal"],
           "branchial": c["branchial"], "device_ms": dev_ms,
           "events_per_s": c["events"] / (dev_ms / 1e3), "e2e_ms": e2e_ms,
           "e2e_events_per_s": c["events"] / (e2e_ms / 1e3)}
    ref = reference_c1_sweep()
    if ref:
        out["reference"] = ref
        out["same_config"] = ref["events"] == c["events"]
        out["e2e_vs_reference_best"] = ref["best"]["ms"] / e2e_ms
        out["e2e_vs_reference_1_thread"] = ref["one_thread"]["ms"] / e2e_ms
        out["device_vs_reference_best"] = ref["best"]["ms"] / dev_ms
    return out


def c3_forwarding(eng, stream, flush, reps=10):
    """C3 (6 levels) with incremental match forwarding off (0), on for every eligible state (1)
    and on for states of >= 48 edges (2): device time and exact equality of the results."""
    import numpy as np
    from hypergraphrewritingengine_b200 import api
    from hypergraphrewritingengine_b200 import workloads as W
    ev = W.config3(6)
    out = {"workload": C3_WORKLOAD, "modes": []}
    base = None
    try:
        for mode in (0, 1, 2):
            eng.set_option(api.OPT_FORWARDING, mode)
            ms, c = _device_ms(eng, stream, flush, ev, reps)
            keys = eng.evolve(ev.rules, ev.roots, ev.steps, quotient=True).keys()
            if base is None:
                base = keys
            same = all(np.array_equal(keys[k], base[k]) for k in keys)
            out["modes"].append({"forwarding": mode, "device_ms": ms,
                                 "events_per_s": c["events"] / (ms / 1e3),
                                 "unique_states_per_s": c["states"] / (ms / 1e3),
                                 "events": c["events"], "unique_states": c["states"],
                                 "identical_to_forwarding_off": same})
    finally:
        eng.set_option(api.OPT_FORWARDING, 0)
    return out


def sharded_batch(eng, dist, world, rank, barrier, per_rank=1024):
    """The batched workload split over the ranks with no exchange step (weak scaling: 1024
    random evolutions per rank, size-balanced by the engine's byte estimate, one engine per
    GPU), counts read back; time = max over ranks of the batch's wall time."""
    import torch
    from hypergraphrewritingengine_b200 import api, shard
    from hypergraphrewritingengine_b200 import workloads as W
    evs = W.config4(n=per_rank * world)
    idx, mine = shard.local_share(evs, rank, world)
    jobs, keep = eng.make_jobs(mine)
    out = (api.ctypes.c_void_p * max(len(mine), 1))()
    eng.set_option(api.OPT_READBACK, 0)
    try:
        ts = []
        for i in range(3):
            barrier()
            t0 = time.perf_counter()
            if mine:
                api._check(eng._L.hgx_evolve_batch(eng._h, jobs, len(mine), out))
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            events = sum(int(eng._L.hgx_result_count(out[k], 1)) for k in range(len(mine)))
            for k in range(len(mine)):
                eng._L.hgx_result_free(out[k])
    finally:
        eng.set_option(api.OPT_READBACK, 1)
    t = max_over_ranks(dist, min(ts[1:]))
    tot = torch.tensor([float(events), float(len(mine))], dtype=torch.float64, device="cuda")
    dist.all_reduce(tot)
    return {"workload": f"c4 split over {world} ranks: {per_rank} random evolutions per rank "
                        "(seed 0x5EED, cap 4096 states each), size-balanced by the byte estimate, "
                        "no exchange step", "scaling": "weak", "evolutions": int(tot[1].item()),
            "events": int(tot[0].item()), "ms_max_over_ranks": t * 1e3,
            "events_per_s": tot[0].item() / t}


def join_index_ab(eng, reps=3):
    """The join with and without its vertex / signature indices (states past 96 edges), on the
    batched workload (C4) and on a batch of large-state evolutions (256 draws of the same
    generator with 65-256 initial edges, 2-4 steps, cap 4096): device time of the warp-per-child
    expand kernel (the large-state path) and wall time of the whole batch, best of `reps`."""
    from hypergraphrewritingengine_b200 import api
    from hypergraphrewritingengine_b200 import workloads as W
    work = {"c4": W.config4(n=1024),
            "large": [W.random_evolution(i, seed=0x1A26E, edges_lo=65, edges_hi=256, steps_lo=2,
                                         steps_hi=4) for i in range(256)]}
    out = {}
    eng.set_option(api.OPT_READBACK, 0)
    eng.set_option(api.OPT_TIMING, 1)
    try:
        for name, evs in work.items():
            jobs, keep = eng.make_jobs(evs)
            row = {}
            for index in (0, 1):
                eng.set_option(api.OPT_JOIN_INDEX, index)
                best = None
                for _ in range(reps + 1):
                    outs = (api.ctypes.c_void_p * len(evs))()
                    t0 = time.perf_counter()
                    api._check(eng._L.hgx_evolve_batch(eng._h, jobs, len(evs), outs))
                    dt = time.perf_counter() - t0
                    ev_total = sum(int(eng._L.hgx_result_count(outs[i], 1)) for i in range(len(evs)))
                    for i in range(len(evs)):
                        eng._L.hgx_result_free(outs[i])
                    st, _ = eng.stage_times()
                    xs = eng.expand_stats()
                    cur = {"wall_ms": dt * 1e3, "device_ms": st["total"], "count_ms": st["count"],
                           "warp_expand_ms": xs["warp_ns"] / 1e6, "events": ev_total}
                    best = cur if best is None or cur["wall_ms"] < best["wall_ms"] else best
                row["index_on" if index else "index_off"] = best
            out[name] = row
    finally:
        eng.set_option(api.OPT_JOIN_INDEX, 1)
        eng.set_option(api.OPT_TIMING, 0)
        eng.set_option(api.OPT_READBACK, 1)
    return out


def batched_vs_plain(eng, n=1024, max_states=4096):
    """1024 random evolutions: one batched pipeline vs. one call per evolution (device-resident,
    counts read back); then both once more with results read back, compared exactly per
    evolution (state-hash set, event / causal / branchial key multisets)."""
    import torch
    from hypergraphrewritingengine_b200 import api
    from hypergraphrewritingengine_b200 import workloads as W
    evs = W.config4(n=n, max_states=max_states)
    jobs, keep = eng.make_jobs(evs)
    eng.set_option(api.OPT_READBACK, 0)
    try:
        # warm-up both paths
        out = (api.ctypes.c_void_p * n)()
        api._check(eng._L.hgx_evolve_batch(eng._h, jobs, n, out))
        for i in range(n):
            eng._L.hgx_result_free(out[i])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        api._check(eng._L.hgx_evolve_batch(eng._h, jobs, n, out))
        t_batch = time.perf_counter() - t0
        batch_counts = []
        for i in range(n):
            batch_counts.append(tuple(int(eng._L.hgx_result_count(out[i], w)) for w in range(6)))
            eng._L.hgx_result_free(out[i])
        t0 = time.perf_counter()
        plain_counts = []
        for i in range(n):
            one = (api.ctypes.c_void_p * 1)()
            api._check(eng._L.hgx_evolve_batch(eng._h, api.ctypes.byref(jobs[i]), 1, one))
            plain_counts.append(tuple(int(eng._L.hgx_result_count(one[0], w)) for w in range(6)))
            eng._L.hgx_result_free(one[0])
        t_plain = time.perf_counter() - t0
    finally:
        eng.set_option(api.OPT_READBACK, 1)
    events = sum(c[1] for c in batch_counts)
    states = sum(c[0] for c in batch_counts)
    # exact comparison, untimed: every evolution's result read back on both paths
    batch_res = eng.evolve_batch(evs, jobs)
    same = batch_counts == plain_counts
    for i in range(n):
        one = eng.evolve_batch([evs[i]], None)[0]
        same = same and one.same_as(batch_res[i])
    return {"workload": f"c4: {n} random evolutions (seed 0x5EED; LHS 2-3, RHS 3-4, arity 2|3, "
                        f"0-2 fresh, 4-64 initial edges, 3-7 steps, WL quotient, cap {max_states} "
                        "states each)",
            "max_states_per_evolution": max_states,
            "events": events, "unique_states": states,
            "batched_events_per_s": events / t_batch, "plain_events_per_s": events / t_plain,
            "batched_ms": t_batch * 1e3, "plain_ms": t_plain * 1e3,
            "speedup_vs_plain": t_plain / t_batch,
            "identical_outputs": bool(same),
            "identical_outputs_compares": "counts, WL class-hash sets and event/causal/branchial "
                                          "key multisets of every evolution"}


def served_vs_plain(eng, n=400, rates=(100.0, 1000.0, 3000.0, 10000.0, float("inf"))):
    """Poisson stream of random evolve requests (initial edges lognormal, median 16, max 256;
    2-8 steps; WL quotient, cap 4096 states), served with continuous batching vs. one request per
    call in arrival order, at arrival rates up to saturation (inf = all requests at t=0)."""
    from hypergraphrewritingengine_b200 import workloads as W
    from hypergraphrewritingengine_b200.serve import Server, serve_plain, summarize
    out = {"workload": f"c5: {n} requests per rate, seed 0xC0FFEE, lognormal initial edges "
                       "(median 16, max 256), 2-8 steps, WL quotient, cap 4096 states; "
                       "admission by estimated device bytes <= 140 GB; per arm the shorter of "
                       "two real-time runs",
           "rates": []}
    for rate in rates:
        stream = W.config5_stream(n, rate_per_s=rate if rate != float("inf") else 1e12,
                                  seed=0xC0FFEE, max_states=4096)
        if rate == float("inf"):
            stream = [(0.0, ev) for _, ev in stream]
        # warm-up, untimed: both arms once over the stream (the engine's arrays and the
        # page-locked result blocks reach their working sizes, as in a long-running server)
        Server(eng).run(stream, realtime=False, admit_per_step=len(stream))
        serve_plain(eng, stream, realtime=False)
        # two real-time runs per arm, alternating; each arm's shorter makespan is kept (the first
        # real-time run of a process can stall on one-off host allocations)
        runs_s, runs_p = [], []
        for _ in range(2):
            runs_s.append(Server(eng).run(stream, realtime=True))
            runs_p.append(serve_plain(eng, stream, realtime=True))
        served = min(runs_s, key=lambda r: summarize(r)["makespan_ms"])
        plain = min(runs_p, key=lambda r: summarize(r)["makespan_ms"])
        same = all(a.result.num_classes == b.result.num_classes and a.result.same_as(b.result)
                   for a, b in zip(served, plain))
        ss, sp = summarize(served), summarize(plain)
        out["rates"].append({"arrivals_per_s": rate if rate != float("inf") else "all at t=0",
                             "served": ss, "plain": sp,
                             "throughput_speedup": ss["events_per_s"] / sp["events_per_s"],
                             "identical_outputs": bool(same),
                             "identical_outputs_compares": "WL class-hash sets and event/causal/"
                                                           "branchial key multisets per request"})
    return out


if __name__ == "__main__":
    main()
