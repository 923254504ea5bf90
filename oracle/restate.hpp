// CPU restatement of the multiway evolution step -- TEST INFRASTRUCTURE ONLY.
//
// This is the oracle the CUDA path is checked against. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg may load it, and only as the checker. The product library
// never links or calls it.
//
// Pinned against the reference engine itself: tests/golden/ holds fixtures produced by
// oracle/_ref/hgref (the reference CPU engine compiled from its own sources), and
// tests/test_oracle_golden.py checks this restatement against every one of them.
//
// Each function cites the reference file:line whose semantics it restates. The code is written
// from the algorithm, not translated: containers, loop structure and sort routines are this
// file's own; what must agree bit for bit is the arithmetic (FNV/mix constants and the order in
// which values enter each fold).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hgx_oracle {

constexpr uint32_t kNone = 0xFFFFFFFFu;

struct Rule {
    std::vector<std::vector<uint8_t>> lhs, rhs;
    uint32_t lhs_mask = 0, rhs_mask = 0, new_mask = 0;
    std::vector<uint8_t> schedule;   // order in which LHS positions are bound
};

struct Event {
    uint32_t in_state, out_state, rule, step;
    uint64_t out_hash;
    std::vector<uint32_t> consumed;   // pattern order
    std::vector<uint32_t> produced;   // RHS order
};

struct Result {
    // states[i]: WL hash and depth. In full multiway every raw state is listed; in quotient
    // mode only the class representatives are.
    std::vector<uint64_t> state_hash;
    std::vector<uint32_t> state_depth;
    std::vector<Event> events;
    std::vector<uint32_t> causal;      // triples (producer, consumer, edge), flattened
    std::vector<uint32_t> branchial;   // pairs (a, b), a < b, flattened
    uint64_t num_classes = 0;
    bool truncated = false;
};

// Pure WL hash of one state given as edges in ascending edge-id order.
uint64_t wl_hash(const std::vector<std::vector<uint32_t>>& edges);

Rule make_rule(const std::vector<std::vector<uint8_t>>& lhs,
               const std::vector<std::vector<uint8_t>>& rhs);

// Transitive reduction of a causal triple list (producer, consumer, edge), flattened: keeps the
// triples whose (producer, consumer) pair is not implied by a path of two or more pairs.
// Restates the unique reduction of the stored relation, hgcommon::tr_reduce
// (common/include/hgcommon/transitive_reduction.hpp:36-94), as read by
// CausalGraph::for_each_causal_edge (hypergraph/include/hypergraph/causal_graph.hpp:295-305).
std::vector<uint32_t> reduce_causal(const std::vector<uint32_t>& triples);

Result evolve(const std::vector<Rule>& rules,
              const std::vector<std::vector<std::vector<uint32_t>>>& roots, uint32_t steps,
              bool quotient, uint64_t max_states);

}  // namespace hgx_oracle
