"""Seeded synthetic workloads for the multiway evolution step.

The five workload shapes are fixed by the benchmark definition: three named single
evolutions, a batch of 1024 random evolutions and a Poisson request stream drawn from the
same generator.  Everything here is deterministic in its seed (splitmix64), so the CUDA
path, the oracle and the reference engine can be given byte-identical inputs.

Rules are ``(lhs, rhs)`` pairs of edge lists over pattern variables (variables numbered by
first appearance in the LHS, fresh variables after them); states are lists of edges over
vertex ids.  This is the same shape ``make_rule(i).lhs(...).rhs(...)`` builds in the
reference (hypergraph/include/hypergraph/pattern.hpp:142-213).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 stream (Steele, Lea & Flood 2014)."""

    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        return self.next() % n

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


@dataclass
class Evolution:
    """One evolve request: rules, root states, step count and exploration mode."""

    rules: list
    roots: list
    steps: int
    quotient: bool = True
    max_states: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)


# --- the three named evolutions --------------------------------------------------------------

def config1() -> Evolution:
    """Binary rule {{x,y},{y,z}} -> {{x,y},{y,z},{z,x}} on a triangle, 5 steps, full multiway."""
    return Evolution(rules=[([[0, 1], [1, 2]], [[0, 1], [1, 2], [2, 0]])],
                     roots=[[[1, 2], [2, 3], [3, 1]]], steps=5, quotient=False,
                     name="c1-triangle-5step-full")


def config2(steps: int = 8, max_states: int = 2_000_000) -> Evolution:
    """{{x,y},{x,z}} -> {{x,z},{x,w},{y,w},{z,w}} from {{1,1},{1,1}}, WL quotient, <= 2M states."""
    return Evolution(rules=[([[0, 1], [0, 2]], [[0, 2], [0, 3], [1, 3], [2, 3]])],
                     roots=[[[1, 1], [1, 1]]], steps=steps, quotient=True,
                     max_states=max_states, name=f"c2-wpp-{steps}step-wlquotient")


def config3(steps: int = 6) -> Evolution:
    """Ternary {{x,y,z},{z,u,v}} -> {{w,w,y},{w,x,u},{v,u,z},{y,v,w}} from two self-loops."""
    return Evolution(rules=[([[0, 1, 2], [2, 3, 4]], [[5, 5, 1], [5, 0, 3], [4, 3, 2], [1, 4, 5]])],
                     roots=[[[1, 1, 1], [1, 1, 1]]], steps=steps, quotient=True,
                     name=f"c3-ternary-{steps}step-wlquotient")


# --- random evolutions (batched and served workloads) ----------------------------------------

def random_rule(rng: SplitMix64, arity: int):
    """Connected random rule: LHS 2-3 edges, RHS 3-4 edges, 0-2 fresh vertices."""
    n_lhs = 2 + rng.below(2)
    n_rhs = 3 + rng.below(2)
    n_fresh = rng.below(3)
    nvars = 0
    lhs = []
    for k in range(n_lhs):
        e = []
        link = rng.below(arity) if k > 0 else -1
        for p in range(arity):
            if p == link:
                e.append(rng.below(nvars))              # shares a variable with an earlier edge
            elif nvars == 0 or rng.below(10) < 6:
                e.append(nvars)
                nvars += 1
            else:
                e.append(rng.below(nvars))
        lhs.append(e)
    pool = list(range(nvars)) + list(range(nvars, nvars + n_fresh))
    rhs = [[pool[rng.below(len(pool))] for _ in range(arity)] for _ in range(n_rhs)]
    # every fresh variable occurs at least once
    for f in range(nvars, nvars + n_fresh):
        if not any(f in e for e in rhs):
            rhs[rng.below(n_rhs)][rng.below(arity)] = f
    return lhs, rhs


def random_hypergraph(rng: SplitMix64, n_edges: int, arity: int):
    """Connected random hypergraph: a spanning chain over 1..N, then uniform random edges."""
    n_vertices = max(3, (n_edges + 1) // 2)
    edges = []
    for j in range(1, n_vertices):
        if len(edges) == n_edges:
            break
        e = [j, j + 1] + [1 + rng.below(n_vertices) for _ in range(arity - 2)]
        edges.append(e)
    while len(edges) < n_edges:
        edges.append([1 + rng.below(n_vertices) for _ in range(arity)])
    return edges


def random_evolution(index: int, seed: int = 0x5EED, max_states: int = 4096,
                     edges_lo: int = 4, edges_hi: int = 64, steps_lo: int = 3,
                     steps_hi: int = 7, lognormal_median: float = 0.0,
                     lognormal_max: int = 0) -> Evolution:
    rng = SplitMix64(seed + index)
    arity = 2 + rng.below(2)
    rule = random_rule(rng, arity)
    if lognormal_median > 0:
        # Box-Muller normal -> lognormal with the requested median, clipped to [edges_lo, max]
        u1 = max(rng.uniform(), 1e-12)
        u2 = rng.uniform()
        z = math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
        n_edges = int(round(lognormal_median * math.exp(0.75 * z)))
        n_edges = min(max(n_edges, edges_lo), lognormal_max or edges_hi)
    else:
        n_edges = edges_lo + rng.below(edges_hi - edges_lo + 1)
    init = random_hypergraph(rng, n_edges, arity)
    steps = steps_lo + rng.below(steps_hi - steps_lo + 1)
    return Evolution(rules=[rule], roots=[init], steps=steps, quotient=True,
                     max_states=max_states, name=f"rand-{index}",
                     meta={"arity": arity, "n_edges": n_edges})


def config4(n: int = 1024, max_states: int = 4096, seed: int = 0x5EED):
    """Batched workload: n independent random evolutions of uneven size."""
    return [random_evolution(i, seed=seed, max_states=max_states) for i in range(n)]


def config5_stream(n_requests: int, rate_per_s: float, seed: int = 0xC0FFEE,
                   max_states: int = 4096):
    """Served workload: Poisson arrivals of random evolve requests.

    Initial edge count is lognormal (median 16, max 256); steps uniform in 2-8.
    Returns a list of (arrival_time_s, Evolution).
    """
    rng = SplitMix64(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += -math.log(max(rng.uniform(), 1e-12)) / rate_per_s
        ev = random_evolution(i, seed=seed ^ 0xA5A5A5A5, max_states=max_states, edges_lo=4,
                              steps_lo=2, steps_hi=8, lognormal_median=16.0, lognormal_max=256)
        out.append((t, ev))
    return out
