// The header-only C++ drop-ins (include/hgx/compat.hpp) driven with the reference's call
// sequence; exit 0 when the counts are the reference engine's (config 1 at 5 steps) and the
// oracle's (config 2 quotient at 5 steps). Needs a GPU.
#include <cstdio>

#include "hgx/compat.hpp"

int main() {
    using namespace hgx::compat::engine;
    Hypergraph hg;
    ParallelEvolutionEngine engine(&hg, 8);
    engine.add_rule(make_rule(0).lhs({0, 1}).lhs({1, 2}).rhs({0, 1}).rhs({1, 2}).rhs({2, 0}).build());
    engine.set_transitive_reduction(false);
    engine.evolve({{1, 2}, {2, 3}, {3, 1}}, 5);
    const auto cg = hg.causal_graph();
    std::printf("c1: states %u events %u classes %zu causal %zu branchial %zu\n", hg.num_states(),
                hg.num_events(), hg.num_canonical_states(), cg.get_causal_edges().size(),
                cg.get_branchial_edges().size());
    bool ok = hg.num_states() == 22204 && hg.num_events() == 22203 && hg.num_canonical_states() == 20 &&
              cg.get_causal_edges().size() == 42816 && cg.get_branchial_edges().size() == 78045;

    // the same evolution with the causal graph reduced transitively (reference: 31,188 triples)
    Hypergraph hg2;
    ParallelEvolutionEngine engine2(&hg2, 8);
    engine2.add_rule(make_rule(0).lhs({0, 1}).lhs({1, 2}).rhs({0, 1}).rhs({1, 2}).rhs({2, 0}).build());
    engine2.set_transitive_reduction(true);
    engine2.evolve({{1, 2}, {2, 3}, {3, 1}}, 5);
    std::printf("c1 reduced: causal %zu\n", hg2.causal_graph().get_causal_edges().size());
    ok = ok && hg2.causal_graph().get_causal_edges().size() == 31188;

    hgx::compat::gpu::EvolveInput in;
    in.rules.push_back({{{0, 1}, {0, 2}}, {{0, 2}, {0, 3}, {1, 3}, {2, 3}}, 3, 4});
    in.initial_state = {{1, 1}, {1, 1}};
    in.num_steps = 5;
    in.explore_from_canonical_states_only = true;
    const auto r = hgx::compat::gpu::evolve(in);
    std::printf("c2: states %zu events %zu classes %llu\n", r.states.size(), r.events.size(),
                (unsigned long long)r.num_classes);
    ok = ok && r.states.size() == 1952 && r.events.size() == 5056 && r.num_classes == 1952;
    // edge contents always; edge ids only under edge_identity (the reference's defaults)
    ok = ok && r.state_edge_ids.empty() && r.states[1951].edges.size() == 12;
    in.edge_identity = true;
    const auto r2 = hgx::compat::gpu::evolve(in);
    bool ids_ok = r2.state_edge_ids.size() == r2.states.size();
    for (size_t s = 0; ids_ok && s < r2.states.size(); ++s)
        ids_ok = r2.state_edge_ids[s].size() == r2.states[s].edges.size() &&
                 r2.states[s].edges == r.states[s].edges;
    std::printf("c2 edge identity: %s\n", ids_ok ? "ids match contents" : "MISMATCH");
    ok = ok && ids_ok;
    bool threw = false;
    try {
        make_rule(0).lhs({0, 40});
    } catch (const std::length_error&) {
        threw = true;
    }
    ok = ok && threw;

    // the rest of the hg_gpu surface: Engine, PersistentEvolver, sizing, modes, refusals
    namespace G = hgx::compat::gpu;
    const G::EngineConfig cfg = G::config_from_input(in);
    G::EngineConfig bigger = cfg;
    bigger.max_states *= 2;
    const bool sizing = cfg.max_states >= (1u << 14) &&
                        G::estimated_device_bytes(bigger) > G::estimated_device_bytes(cfg);
    G::PersistentEvolver pe;
    const auto p1 = pe.run(in);
    const auto p2 = pe.run(in);   // the same engine, reused
    const bool persistent = pe.has_engine() && p1.states.size() == 1952 && p2.events.size() == 5056 &&
                            !pe.run_session(in, nullptr, 0).ok;
    G::EvolveInput full = in;     // canonicalization None: every state its own class
    full.rules = {{{{0, 1}, {1, 2}}, {{0, 1}, {1, 2}, {2, 0}}, 3, 3}};
    full.initial_state = {{1, 2}, {2, 3}, {3, 1}};
    full.canonicalization = G::CanonicalizationMode::None;
    full.transitive_reduction = false;
    full.edge_identity = false;
    const auto rf = G::evolve(full);
    const bool none_mode = rf.states.size() == 22204 && rf.events.size() == 22203 &&
                           rf.observable_num_branchial() == 78045;
    G::EvolveInput two = in;      // two isomorphic roots collapse under quotient_initial_states
    two.initial_states = {{{1, 1}, {1, 1}}, {{5, 5}, {5, 5}}};
    two.num_steps = 2;
    const auto t_sep = G::evolve(two);
    two.quotient_initial_states = true;
    const auto t_one = G::evolve(two);
    G::EvolveInput single = two;
    single.initial_states = {{{1, 1}, {1, 1}}};
    const auto t_single = G::evolve(single);
    const bool roots_ok = t_one.events.size() == t_single.events.size() &&
                          t_one.states.size() == t_single.states.size() &&
                          t_sep.events.size() > t_one.events.size();
    G::EvolveInput capped = in;   // a device-memory ceiling below what the run needs
    capped.max_device_memory_bytes = 4096;
    const auto rc = G::evolve(capped);
    const bool oom = rc.states.empty() && !rc.warnings.empty() &&
                     rc.warnings[0].kind == G::ErrorKind::kDeviceOutOfMemory;
    bool sampling_refused = false;
    try {
        G::EvolveInput s2 = in;
        s2.exploration_probability = 0.5f;
        G::evolve(s2);
    } catch (const std::invalid_argument&) {
        sampling_refused = true;
    }
    std::printf("hg_gpu: sizing %d persistent %d none-mode %d roots %zu/%zu oom %d sampling refused %d\n",
                sizing, persistent, none_mode, t_sep.events.size(), t_one.events.size(), oom,
                sampling_refused);
    ok = ok && sizing && persistent && none_mode && roots_ok && oom && sampling_refused;
    std::printf(ok ? "compat ok\n" : "compat MISMATCH\n");
    return ok ? 0 : 1;
}
