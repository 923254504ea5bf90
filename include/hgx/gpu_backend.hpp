// hgx/gpu_backend.hpp -- the worker's GPU backend: a parsed job in, the WXF reply out. Header
// only, over hgx/hg_gpu.hpp.
//
// Replaces run_gpu_evolution(const GpuJob&, const HostBridge&) of the reference
// (paclet_source/hg_gpu_backend.hpp:119, hg_gpu_backend.cpp:25-829), which run_rewriting_core
// routes GPU jobs to. The job type carries the reference's GpuJob fields under the same names
// (hgx::compat::GpuJob below); run_gpu_evolution_with() is a template, so the reference's own
// GpuJob and HostBridge can be passed unchanged.
//
// The reply is the association the reference emits, in its key order -- States, Events,
// CausalEdges, BranchialEdges, GlobalEdges, StateBitvectors, NumStates, NumEvents,
// NumCausalEdges, NumBranchialEdges, Warnings -- with one difference of substance: states are
// grouped by the WL canonical hash the device computed (state mode Full), by exact edge content
// (Automatic) or not at all (None), where the reference regroups them by an IR hash it
// recomputes on the host (hg_gpu_backend.cpp:269-315). A class's Edges are its representative's
// own labels (the IR canonical relabelling is not computed), and CanonicalHash carries the WL hash.
// Not provided, and refused with an exception rather than answered in another shape: session
// verbs other than Evolve, graph properties (GraphData), and the branchial state-edge views.
#pragma once
#include <cstdint>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "hg_gpu.hpp"
#include "wxf.hpp"

namespace hgx {
namespace compat {

// paclet_source/hg_core.hpp: progress reporting from the evolution core (may be empty).
struct HostBridge {
    std::function<void(const std::string&)> progress;
};

// paclet_source/hg_gpu_backend.hpp:15-110: a parsed evolution job, field for field.
struct GpuJob {
    const std::vector<std::pair<std::string, std::vector<std::vector<std::vector<int64_t>>>>>& rules;
    const std::vector<std::vector<std::vector<int64_t>>>& initial_states;
    // The two mode codes have different orders (as in the reference).
    struct EventCanonCode { static constexpr int kNone = 0, kFull = 1, kAutomatic = 2; };
    struct StateCanonCode { static constexpr int kNone = 0, kAutomatic = 1, kFull = 2; };
    int steps = 0;
    int event_canon_mode = EventCanonCode::kNone;
    int state_canon_mode = StateCanonCode::kFull;
    bool transitive_reduction = true;
    bool explore_from_canonical_states_only = false;
    bool quotient_initial_states = false;
    double exploration_probability = 1.0;
    uint64_t random_seed = 0;
    uint64_t max_device_memory_bytes = 0;
    double transition_rate = 1.0;
    std::vector<double> rule_weights;
    uint64_t max_states_per_step = 0;
    uint64_t max_successor_states_per_parent = 0;
    uint64_t matches_per_state_rule = 0;
    bool include_states = true;
    bool include_events = true;
    bool include_events_minimal = false;
    bool include_causal_edges = true;
    bool include_branchial_edges = true;
    bool include_canonical_hashes = false;
    bool include_num_states = true;
    bool include_num_events = true;
    bool include_num_causal_edges = true;
    bool include_num_branchial_edges = true;
    bool include_branchial_state_edges = false;
    bool include_branchial_state_edges_all_siblings = false;
    bool include_global_edges = false;
    bool include_state_bitvectors = false;
    std::vector<std::string> graph_properties;
    bool edge_deduplication = true;
    int branchial_step = 0;
    bool show_genesis_events = false;
    std::string session_op;
    uint64_t session_handle = 0;
    std::vector<int64_t> session_from;
};

namespace backend_detail {

// The job as an hg_gpu::EvolveInput: rule variables checked (0..31) before narrowing, empty edges
// dropped, an empty LHS refused; each root's vertex labels (any int64) renumbered densely in
// order of first appearance; modes decoded from their codes; what to record derived from what
// the reply will carry.
template <class Job>
gpu::EvolveInput build_input(const Job& job) {
    gpu::EvolveInput in;
    size_t index = 0;
    for (const auto& named : job.rules) {
        const auto& sides = named.second;
        if (sides.size() != 2)
            throw std::runtime_error("rule " + std::to_string(index) + " must have a left and a right "
                                     "side (got " + std::to_string(sides.size()) + " parts)");
        gpu::RewriteRule r;
        int64_t top[2] = {-1, -1};
        for (int side = 0; side < 2; ++side) {
            const char* name = side == 0 ? "LHS" : "RHS";
            for (const auto& edge : sides[side]) {
                std::vector<uint8_t> e;
                for (int64_t v : edge) {
                    if (v < 0)
                        throw std::runtime_error("rule " + std::to_string(index) + " " + name +
                                                 " has a negative pattern variable");
                    if (v >= static_cast<int64_t>(gpu::MAX_VARS))
                        throw std::runtime_error("rule " + std::to_string(index) + " " + name +
                                                 " uses pattern variable " + std::to_string(v) +
                                                 ", but the maximum is " +
                                                 std::to_string(gpu::MAX_VARS - 1));
                    e.push_back(static_cast<uint8_t>(v));
                    top[side] = std::max<int64_t>(top[side], v);
                }
                if (e.empty()) continue;
                (side == 0 ? r.lhs : r.rhs).push_back(std::move(e));
            }
        }
        if (r.lhs.empty())
            throw std::runtime_error("rule " + std::to_string(index) + " has an empty left-hand side");
        r.num_lhs_vars = static_cast<uint8_t>(top[0] + 1);
        r.num_rhs_vars = static_cast<uint8_t>(top[1] + 1);
        in.rules.push_back(std::move(r));
        ++index;
    }
    for (const auto& state : job.initial_states) {
        std::unordered_map<int64_t, gpu::VertexId> ids;
        std::vector<std::vector<gpu::VertexId>> edges;
        for (const auto& edge : state) {
            std::vector<gpu::VertexId> e;
            for (int64_t v : edge)
                e.push_back(ids.emplace(v, static_cast<gpu::VertexId>(ids.size())).first->second);
            if (!e.empty()) edges.push_back(std::move(e));
        }
        if (!edges.empty()) in.initial_states.push_back(std::move(edges));
    }
    in.num_steps = static_cast<uint32_t>(job.steps > 0 ? job.steps : 0);
    in.canonicalization = job.state_canon_mode == 0   ? gpu::CanonicalizationMode::None
                          : job.state_canon_mode == 1 ? gpu::CanonicalizationMode::Automatic
                                                      : gpu::CanonicalizationMode::Full;
    in.event_canonicalization = job.event_canon_mode == 1   ? gpu::EventCanonicalizationMode::Full
                                : job.event_canon_mode == 2 ? gpu::EventCanonicalizationMode::Automatic
                                                            : gpu::EventCanonicalizationMode::None;
    in.record.causal = job.include_causal_edges || job.include_num_causal_edges;
    in.record.branchial = job.include_branchial_edges || job.include_num_branchial_edges ||
                          job.include_branchial_state_edges;
    in.record.raw_events = job.include_events || job.include_num_events ||
                           job.include_branchial_state_edges ||
                           job.include_branchial_state_edges_all_siblings || job.show_genesis_events;
    in.transitive_reduction = job.transitive_reduction;
    in.explore_from_canonical_states_only = job.explore_from_canonical_states_only;
    in.quotient_initial_states = job.quotient_initial_states;
    in.exploration_probability = static_cast<float>(job.exploration_probability);
    in.exploration_seed = job.random_seed;
    in.transition_rate = job.transition_rate;
    in.rule_weights = job.rule_weights;
    in.max_states_per_step = static_cast<uint32_t>(job.max_states_per_step);
    in.max_successor_states_per_parent = static_cast<uint32_t>(job.max_successor_states_per_parent);
    in.matches_per_state_rule = static_cast<uint32_t>(job.matches_per_state_rule);
    in.edge_identity = job.include_global_edges || job.include_state_bitvectors || job.show_genesis_events;
    in.max_device_memory_bytes = job.max_device_memory_bytes;
    return in;
}

inline void write_edges(wxf::Writer& w, const std::vector<std::vector<gpu::VertexId>>& edges) {
    w.list(edges.size());
    int64_t idx = 0;
    for (const auto& e : edges) {
        w.list(e.size() + 1);
        w.integer(idx++);
        for (auto v : e) w.integer(static_cast<int64_t>(v));
    }
}

inline void write_id_list(wxf::Writer& w, const std::vector<gpu::EdgeId>& ids) {
    size_t n = 0;
    for (auto x : ids) n += x != gpu::INVALID_ID ? 1 : 0;
    w.list(n);
    for (auto x : ids)
        if (x != gpu::INVALID_ID) w.integer(static_cast<int64_t>(x));
}

}  // namespace backend_detail

// Run the job on the GPU and return the WXF reply (see the file comment). Throws std::exception
// on error, as the reference does.
template <class Job, class Bridge>
std::vector<uint8_t> run_gpu_evolution_with(gpu::PersistentEvolver& evolver, const Job& job,
                                            const Bridge& host) {
    using namespace backend_detail;
    const std::string& op = job.session_op;
    if (!op.empty() && op != "Evolve")
        throw std::runtime_error("Op '" + op + "': sessions (Open, Step, Query, Close) are not "
                                 "provided on this GPU path; use 'Evolve'");
    if (!job.graph_properties.empty())
        throw std::runtime_error("graph properties (GraphData) are not built by this GPU backend");
    if (job.include_branchial_state_edges || job.include_branchial_state_edges_all_siblings)
        throw std::runtime_error("BranchialStateEdges views are not built by this GPU backend");

    const gpu::EvolveInput in = build_input(job);
    const gpu::EvolveResult result = in.initial_states.empty() ? gpu::EvolveResult{} : evolver.run(in);

    // classes: the key the requested state mode identifies states by; first state = representative
    const auto mode = in.canonicalization;
    std::unordered_map<gpu::StateId, gpu::StateId> rep;   // state -> representative
    std::vector<gpu::StateId> reps;
    {
        std::unordered_map<uint64_t, gpu::StateId> by_hash;
        std::map<std::vector<std::vector<gpu::VertexId>>, gpu::StateId> by_content;
        for (const auto& s : result.states) {
            gpu::StateId r = s.id;
            if (mode == gpu::CanonicalizationMode::Full) {
                r = by_hash.emplace(s.canonical_hash, s.id).first->second;
            } else if (mode == gpu::CanonicalizationMode::Automatic) {
                auto key = s.edges;
                std::sort(key.begin(), key.end());
                r = by_content.emplace(std::move(key), s.id).first->second;
            }
            rep[s.id] = r;
            if (r == s.id) reps.push_back(s.id);
        }
    }
    auto rep_of = [&](gpu::StateId s) -> int64_t {
        auto it = rep.find(s);
        return static_cast<int64_t>(it == rep.end() ? s : it->second);
    };
    // per state: the smallest step of an event producing it; roots are no event's output
    std::unordered_map<gpu::StateId, uint32_t> step_of;
    for (const auto& e : result.events) {
        auto it = step_of.find(e.output_state);
        if (it == step_of.end() || e.step < it->second) step_of[e.output_state] = e.step;
    }
    std::unordered_map<gpu::StateId, const gpu::CanonicalState*> state_by_id;
    for (const auto& s : result.states) state_by_id[s.id] = &s;

    // Genesis events (ShowGenesisEvents): one per initial state, ids above every event id, rule
    // index -1, producing that root's edges; an event consuming an initial edge is caused by it.
    std::vector<gpu::StateId> roots;
    std::unordered_map<gpu::EdgeId, size_t> root_of_edge;
    gpu::StateId genesis_state = 0;
    gpu::EventId first_genesis = 0;
    if (job.show_genesis_events) {
        for (const auto& s : result.states) genesis_state = std::max<gpu::StateId>(genesis_state, s.id + 1);
        for (const auto& e : result.events) first_genesis = std::max<gpu::EventId>(first_genesis, e.id + 1);
        for (const auto& s : result.states) {
            if (step_of.count(s.id)) continue;
            if (s.id < result.state_edge_ids.size())
                for (auto id : result.state_edge_ids[s.id]) root_of_edge[id] = roots.size();
            roots.push_back(s.id);
        }
    }

    // causal pairs, deduplicated by (from, to) as the reference's FFI reports them
    std::vector<std::pair<gpu::EventId, gpu::EventId>> causal;
    {
        std::unordered_set<uint64_t> seen;
        for (const auto& c : result.causal_edges)
            if (seen.insert((uint64_t(c.from) << 32) | c.to).second) causal.push_back({c.from, c.to});
        for (const auto& e : result.events)
            for (auto id : e.consumed_edges) {
                auto it = root_of_edge.find(id);
                if (it == root_of_edge.end()) continue;
                const gpu::EventId from = first_genesis + static_cast<gpu::EventId>(it->second);
                if (seen.insert((uint64_t(from) << 32) | e.id).second) causal.push_back({from, e.id});
            }
    }

    size_t n_keys = 0;
    n_keys += job.include_states + job.include_events + job.include_causal_edges +
              job.include_branchial_edges + job.include_global_edges + job.include_state_bitvectors +
              job.include_num_states + job.include_num_events + job.include_num_causal_edges +
              job.include_num_branchial_edges + (!result.warnings.empty());
    wxf::Writer w;
    w.association(n_keys);

    if (job.include_states) {
        w.key("States");
        w.association(reps.size());
        for (gpu::StateId r : reps) {
            const auto* s = state_by_id[r];
            const bool initial = step_of.find(r) == step_of.end();
            w.int_key(r);
            w.association(6 + (job.include_canonical_hashes ? 1 : 0));
            w.key("Id"); w.integer(r);
            w.key("CanonicalId"); w.integer(r);
            w.key("ContentStateId"); w.integer(r);
            w.key("Step"); w.integer(initial ? 0 : step_of[r]);
            w.key("Edges"); write_edges(w, s->edges);
            w.key("IsInitial"); w.boolean(initial);
            if (job.include_canonical_hashes) {
                w.key("CanonicalHash");
                w.integer(static_cast<int64_t>(s->canonical_hash));
            }
        }
    }
    if (job.include_events) {
        const size_t fields = job.include_events_minimal ? 7 : 9;
        w.key("Events");
        w.association(result.events.size() + roots.size());
        for (const auto& e : result.events) {
            w.int_key(e.id);
            w.association(fields);
            w.key("Id"); w.integer(e.id);
            w.key("CanonicalId");
            w.integer(e.canonical_id == gpu::INVALID_ID ? e.id : e.canonical_id);
            w.key("RuleIndex"); w.integer(e.rule);
            w.key("InputState"); w.integer(e.input_state);
            w.key("OutputState"); w.integer(e.output_state);
            w.key("CanonicalInputState"); w.integer(rep_of(e.input_state));
            w.key("CanonicalOutputState"); w.integer(rep_of(e.output_state));
            if (!job.include_events_minimal) {
                w.key("ConsumedEdges"); write_id_list(w, e.consumed_edges);
                w.key("ProducedEdges"); write_id_list(w, e.produced_edges);
            }
        }
        for (size_t i = 0; i < roots.size(); ++i) {
            const int64_t id = first_genesis + static_cast<int64_t>(i);
            w.int_key(id);
            w.association(fields);
            w.key("Id"); w.integer(id);
            w.key("CanonicalId"); w.integer(id);
            w.key("RuleIndex"); w.integer(-1);
            w.key("InputState"); w.integer(genesis_state);
            w.key("OutputState"); w.integer(roots[i]);
            w.key("CanonicalInputState"); w.integer(genesis_state);
            w.key("CanonicalOutputState"); w.integer(rep_of(roots[i]));
            if (!job.include_events_minimal) {
                w.key("ConsumedEdges"); w.list(0);
                w.key("ProducedEdges");
                write_id_list(w, roots[i] < result.state_edge_ids.size() ? result.state_edge_ids[roots[i]]
                                                                         : std::vector<gpu::EdgeId>{});
            }
        }
    }
    if (job.include_causal_edges) {
        w.key("CausalEdges");
        w.list(causal.size());
        for (const auto& c : causal) {
            w.association(4);
            w.key("From"); w.integer(c.first);
            w.key("To"); w.integer(c.second);
            w.key("RawFrom"); w.integer(c.first);
            w.key("RawTo"); w.integer(c.second);
        }
    }
    if (job.include_branchial_edges) {
        w.key("BranchialEdges");
        w.list(result.branchial_edges.size());
        for (const auto& b : result.branchial_edges) {
            w.association(2);
            w.key("From"); w.integer(b.a);
            w.key("To"); w.integer(b.b);
        }
    }
    if (job.include_global_edges) {
        size_t n = 0;
        for (const auto& vs : result.global_edges) n += vs.empty() ? 0 : 1;
        w.key("GlobalEdges");
        w.list(n);
        for (size_t id = 0; id < result.global_edges.size(); ++id) {
            const auto& vs = result.global_edges[id];
            if (vs.empty()) continue;
            w.list(vs.size() + 1);
            w.integer(static_cast<int64_t>(id));
            for (auto v : vs) w.integer(static_cast<int64_t>(v));
        }
    }
    if (job.include_state_bitvectors) {
        w.key("StateBitvectors");
        w.association(result.state_edge_ids.size());
        for (size_t s = 0; s < result.state_edge_ids.size(); ++s) {
            w.int_key(static_cast<int64_t>(s));
            write_id_list(w, result.state_edge_ids[s]);
        }
    }
    if (job.include_num_states) {
        w.key("NumStates");
        w.integer(static_cast<int64_t>(reps.size()));
    }
    if (job.include_num_events) {
        w.key("NumEvents");
        w.integer(static_cast<int64_t>(result.observable_num_events()));
    }
    if (job.include_num_causal_edges) {
        w.key("NumCausalEdges");
        w.integer(static_cast<int64_t>(causal.size()));
    }
    if (job.include_num_branchial_edges) {
        w.key("NumBranchialEdges");
        w.integer(static_cast<int64_t>(result.observable_num_branchial()));
    }
    if (!result.warnings.empty()) {
        if (host.progress) host.progress("HGEvolve (GPU): capacity limit -- returning partial result");
        w.key("Warnings");
        w.list(result.warnings.size());
        for (const auto& x : result.warnings) {
            w.association(3);
            w.key("Kind"); w.string(gpu::error_kind_name(x.kind));
            w.key("Count"); w.integer(x.count);
            w.key("Context"); w.string(x.context);
        }
    }
    return w.take();
}

// One engine for the process, reused by every job (jobs run one at a time, as in the worker).
inline std::vector<uint8_t> run_gpu_evolution(const GpuJob& job, const HostBridge& host) {
    static gpu::PersistentEvolver evolver;
    return run_gpu_evolution_with(evolver, job, host);
}

}  // namespace compat
}  // namespace hgx
