"""B200-native multiway evolution step (sm_100a CUDA behind a C-ABI).

The native library ``libhgx.so`` is required; there is no CPU fallback.
"""
from .api import (CausalGraph, Engine, EvolveResult, HgxError, Hypergraph, Job,  # noqa: F401
                  ParallelEvolutionEngine, RewriteRule, RuleBuilder, encode_roots, encode_rule,
                  encode_rules, load_library, make_rule)
