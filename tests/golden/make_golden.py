"""Generate the golden fixtures in tests/golden/ by running the reference engine itself.

    make -C oracle ref            # builds oracle/_ref/hgref from the reference's own sources
    python tests/golden/make_golden.py

Full-multiway cases run the reference in WL mode (StateCanonicalizationMode::None, reported WL
canonical hashes, transitive reduction off) and store counts, the sorted WL class hashes, and
FNV digests of the sorted event / causal / branchial key multisets (keys as in the reference's
gpu/tests/test_gpu_vs_cpu_differential.cpp:119-157); small cases also store the full key arrays.

Quotient cases run the reference's quotient exploration serially (its parallel quotient run is
schedule-dependent), which is IR-keyed (Full mode): only the class and event counts are stored.
They pin the WL-quotient path wherever the WL classes coincide with the IR classes, at the depths
where the reference's serial quotient exploration is complete (<= 5 on the named workloads).

Also records the reference's own golden-matrix rows for the None/None/full-multiway mode
(reference/golden_matrix.txt), read as text.

The "tr" section re-runs the full-multiway cases with the causal graph's transitive reduction on
(serial execution) and stores the reduced causal count and key digest. The "evsig" section re-runs
them with event canonicalisation (signature keys 3 = Full and 15 = input|output|step|rule) and
stores the canonical event count and the number of distinct state hashes the reference reports
then (it switches to its exact IR hash when event keys are on, so the counts pin the WL path
wherever IR and WL classes coincide). `python make_golden.py tr` (or `evsig`) recomputes only that
section in the existing golden.json.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
sys.path.insert(0, HERE)

from oracle import pyoracle  # noqa: E402
import cases  # noqa: E402

REF_MATRIX = os.path.join(os.environ.get("HGX_REFERENCE", "/root/reference"),
                          "reference", "golden_matrix.txt")


def tr_section():
    out = {}
    for name, rules, roots, steps in cases.all_full_cases():
        r = pyoracle.run_reference(rules, roots, steps, quotient=False, threads=0, arrays=True,
                                   tr=True)
        entry = {"steps": steps, "causal": r["causal"], "causal_digest": r["causal_digest"]}
        if r["causal"] <= 1500:
            entry["causal_keys"] = r["causal_keys"]
        out[name] = entry
        print("tr", name, r["causal"], f"{r['ms']:.0f}ms", flush=True)
    return out


def evsig_section():
    out = {}
    for name, rules, roots, steps in cases.all_full_cases():
        entry = {"steps": steps}
        for keys in (3, 15):
            r = pyoracle.run_reference(rules, roots, steps, quotient=False, threads=0, evkeys=keys)
            entry[str(keys)] = {"events": r["events"], "raw_events": r["raw_events"],
                                "classes": r["wl_classes"]}
        out[name] = entry
        print("evsig", name, entry["3"], entry["15"], flush=True)
    return out


SECTIONS = {"tr": tr_section, "evsig": evsig_section}


def main():
    if len(sys.argv) == 2 and sys.argv[1] in SECTIONS:
        path = os.path.join(HERE, "golden.json")
        with open(path) as fh:
            out = json.load(fh)
        out[sys.argv[1]] = SECTIONS[sys.argv[1]]()
        with open(path, "w") as fh:
            json.dump(out, fh, indent=0, sort_keys=True)
        return
    out = {"full": {}, "quotient": {}, "matrix": {}}
    for name, rules, roots, steps in cases.all_full_cases():
        r = pyoracle.run_reference(rules, roots, steps, quotient=False, threads=8, arrays=True)
        entry = {k: r[k] for k in ("raw_states", "events", "wl_classes", "causal", "branchial",
                                   "event_digest", "causal_digest", "branchial_digest",
                                   "state_hashes")}
        entry["steps"] = steps
        entry["state_digest"] = pyoracle.digest(r["state_hashes"])
        if len(r["state_hashes"]) > 2000:
            del entry["state_hashes"]
        if r["events"] <= 600 and r["branchial"] <= 1500:
            for k in ("event_keys", "causal_keys", "branchial_keys"):
                entry[k] = r[k]
        out["full"][name] = entry
        print(name, r["events"], r["wl_classes"], f"{r['ms']:.0f}ms", flush=True)
    for name, rules, roots, steps in cases.all_quotient_cases():
        # serial execution: the reference's parallel quotient exploration is schedule-dependent
        r = pyoracle.run_reference(rules, roots, steps, quotient=True, threads=0)
        out["quotient"][name] = {"steps": steps, "raw_states": r["raw_states"], "events": r["events"],
                                 "ir_classes": r["canonical_states"]}
        print(name, r["events"], r["canonical_states"], f"{r['ms']:.0f}ms", flush=True)
    if os.path.exists(REF_MATRIX):
        for line in open(REF_MATRIX):
            f = line.split()
            if len(f) >= 11 and not line.startswith("#") and f[1:4] == ["None", "None", "0"]:
                out["matrix"][f[0]] = {"steps": int(f[4]), "states": int(f[5]), "events": int(f[6]),
                                       "causal": int(f[7]), "pairs": int(f[8]), "branchial": int(f[9])}
    out["tr"] = tr_section()
    out["evsig"] = evsig_section()
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)


if __name__ == "__main__":
    main()
