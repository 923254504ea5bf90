"""Named parity cases: the three named workloads at every depth the reference engine finishes,
the reference's own rule corpus (reference/oracle_corpus.hpp:208-318, with the depths its
golden matrix uses), and edge cases (several roots, unary edges, a deleting rule that reaches the
empty state, duplicate edges, disconnected and self-loop patterns).

Each case: (name, rules, roots, steps, quotient).  rules: list of (lhs, rhs).
"""

C1_RULE = ([[0, 1], [1, 2]], [[0, 1], [1, 2], [2, 0]])
C1_INIT = [[1, 2], [2, 3], [3, 1]]
C2_RULE = ([[0, 1], [0, 2]], [[0, 2], [0, 3], [1, 3], [2, 3]])
C2_INIT = [[1, 1], [1, 1]]
C3_RULE = ([[0, 1, 2], [2, 3, 4]], [[5, 5, 1], [5, 0, 3], [4, 3, 2], [1, 4, 5]])
C3_INIT = [[1, 1, 1], [1, 1, 1]]

# The reference's corpus (name, rules, init, oracle depth).
CORPUS = [
    ("binary-growth", [([[0, 1]], [[0, 2], [1, 2]])], [[0, 1]], 3),
    ("wolfram-2to4", [([[0, 1], [0, 2]], [[0, 1], [0, 3], [1, 3], [2, 3]])], [[0, 1], [0, 2]], 2),
    ("triangle", [([[0, 1], [1, 2]], [[0, 2], [2, 3], [3, 0]])], [[0, 1], [1, 2]], 2),
    ("reductive-2to1", [([[0, 1], [1, 2]], [[0, 2]])], [[0, 1], [1, 2], [2, 3], [3, 4]], 3),
    ("idempotent-2to2", [([[0, 1], [1, 2]], [[0, 2], [2, 1]])], [[0, 1], [1, 2]], 3),
    ("self-loop", [([[0, 0]], [[0, 1], [1, 0]])], [[0, 0]], 3),
    ("mixed-arity", [([[0, 1]], [[0, 1, 2], [2, 0]])], [[0, 1]], 3),
    ("arity3-growth", [([[0, 1, 2]], [[0, 1, 3], [1, 2, 3]])], [[0, 1, 2]], 3),
    ("disconnected-lhs", [([[0, 1], [2, 3]], [[0, 2], [1, 3]])], [[0, 1], [2, 3]], 3),
    ("arity4-growth", [([[0, 1, 2, 3]], [[0, 1, 2, 4], [1, 2, 3, 4]])], [[0, 1, 2, 3]], 3),
    ("mixed-arity-lhs", [([[0, 1], [0, 1, 2]], [[0, 2], [1, 2, 3]])], [[0, 1], [0, 1, 2]], 3),
    ("mixed-arity-init", [([[0, 1]], [[0, 1, 2]])], [[0, 1], [1, 2, 3], [2, 3]], 3),
    ("arity3-to-2", [([[0, 1, 2]], [[0, 1], [1, 2]])], [[0, 1, 2], [1, 2, 3]], 3),
    ("arity1-with-binary", [([[0], [0, 1]], [[1], [0, 1], [0, 2]])], [[0], [0, 1]], 3),
    ("cycle4-automorphic", [([[0, 1], [1, 2]], [[0, 1], [1, 3], [3, 2]])], [[0, 1], [1, 2], [2, 3], [3, 0]], 3),
    ("star4-automorphic", [([[0, 1]], [[0, 1], [1, 2]])], [[0, 1], [0, 2], [0, 3], [0, 4]], 2),
    ("multi-rule", [([[0, 1]], [[0, 2], [1, 2]]), ([[0, 1], [1, 2]], [[0, 2]])], [[0, 1], [1, 2]], 2),
]

EDGE_CASES = [
    # two roots, one of them isomorphic to the other
    ("multi-root", [C1_RULE], [C1_INIT, [[5, 6], [6, 7], [7, 5]], [[1, 2], [2, 3]]], 3),
    # deleting rule: reaches the empty state (reserved hash)
    ("deleting", [([[0, 1]], [])], [[[1, 2], [2, 3]]], 2),
    # unary edges beside binary ones (initial-colour truncation path of the WL core)
    ("unary-heavy", [([[0], [0, 1]], [[0], [0], [0, 1], [1, 2]])], [[[1], [1], [1], [1, 2]]], 3),
    # duplicate edges and a repeated-variable pattern
    ("dup-edges", [([[0, 0], [0, 1]], [[0, 0], [1, 0], [1, 1]])], [[[1, 1], [1, 1], [1, 2]]], 3),
    # cyclic 3-edge LHS
    ("triangle-lhs", [([[0, 1], [1, 2], [2, 0]], [[0, 1], [1, 2], [2, 3], [3, 0]])],
     [[[1, 2], [2, 3], [3, 1], [1, 4], [4, 2]]], 3),
]


def all_full_cases():
    """(name, rules, roots, steps) run in full multiway mode against the reference."""
    out = []
    for s in range(1, 6):
        out.append((f"c1-full-{s}", [C1_RULE], [C1_INIT], s))
    for s in range(1, 5):
        out.append((f"c2-full-{s}", [C2_RULE], [C2_INIT], s))
    for s in range(1, 6):
        out.append((f"c3-full-{s}", [C3_RULE], [C3_INIT], s))
    for name, rules, init, depth in CORPUS:
        out.append((f"corpus-{name}-{depth}", rules, [init], depth))
    for name, rules, roots, depth in EDGE_CASES:
        roots = roots if isinstance(roots[0][0], list) else [roots]
        out.append((f"edge-{name}-{depth}", rules, roots, depth))
    return out


def all_quotient_cases():
    """(name, rules, roots, steps) run in quotient mode (reference: Full/IR keyed)."""
    out = []
    for s in range(1, 6):
        out.append((f"c2-quot-{s}", [C2_RULE], [C2_INIT], s))
    for s in range(1, 6):
        out.append((f"c3-quot-{s}", [C3_RULE], [C3_INIT], s))
    for name, rules, init, depth in CORPUS:
        out.append((f"corpus-{name}-{depth + 1}", rules, [init], depth + 1))
    return out
