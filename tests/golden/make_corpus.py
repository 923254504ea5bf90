"""Fixtures from the reference's shared engine golden corpus (reference/golden_corpus.wl:
MultiwaySystem values at the final step under CanonicalizeStates -> Full, each case's expected
{states, rawEvents, causal, branchial}).

    python tests/golden/make_corpus.py      # reads the reference tree, writes golden_corpus.json

The .wl file is read as text: every case is one association with "name", "rules", "init",
"steps" and "expected". Rules are lists of {lhs, rhs} edge lists whose vertices double as
pattern-variable indices (as in the reference's FFI). The evolution is full multiway (every raw
state expanded), so rawEvents, causal and branchial do not depend on how states are identified;
"states" counts IR isomorphism classes.
"""
import json
import os
import re

REF = os.environ.get("HGX_REFERENCE", "/root/reference")
SRC = os.path.join(REF, "reference", "golden_corpus.wl")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_corpus.json")


def _wl_to_json(text: str):
    """A Wolfram list of integers ({...}) as JSON."""
    return json.loads(text.replace("{", "[").replace("}", "]"))


def parse(text: str):
    cases = []
    for m in re.finditer(r"<\|(.*?)\|>", text, re.S):
        body = m.group(1)
        field = lambda k: re.search(r'"%s"\s*->\s*(.*?)(?=,\s*"\w+"\s*->|\s*$)' % k, body, re.S).group(1)  # noqa: E731
        rules = _wl_to_json(field("rules"))
        cases.append({
            "name": json.loads(field("name")),
            "rules": [[lhs, rhs] for lhs, rhs in rules],
            "init": _wl_to_json(field("init")),
            "steps": int(field("steps")),
            "expected": dict(zip(("states", "raw_events", "causal", "branchial"),
                                 _wl_to_json(field("expected")))),
        })
    return cases


def main():
    cases = parse(open(SRC).read())
    with open(OUT, "w") as fh:
        json.dump({"source": "reference/golden_corpus.wl", "cases": cases}, fh, indent=1)
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
