// hgx/compat.hpp -- header-only C++ surfaces of the reference engine, over the C ABI (hgx.h).
//
// Two drop-ins, each with the reference's names, argument meaning and error behaviour:
//
//   hgx::compat::engine   make_rule(i).lhs(..).rhs(..).build(), Hypergraph,
//                         ParallelEvolutionEngine(&hg, threads).add_rule(r).evolve(init, steps),
//                         hg.num_states() / num_events() / num_canonical_states(),
//                         hg.causal_graph().get_causal_edges() / get_branchial_edges()
//                         (reference: hypergraph/include/hypergraph/pattern.hpp:142-213,
//                          parallel_evolution.hpp:743-1041, hypergraph.hpp:567-811)
//   hgx::compat::gpu      RewriteRule / EvolveInput / EvolveResult, evolve(const EvolveInput&),
//                         Engine, PersistentEvolver, EngineConfig, config_from_input,
//                         estimated_device_bytes (reference: gpu/include/hg_gpu/evolve.hpp;
//                         defined in hgx/hg_gpu.hpp, included at the end of this header)
//
// The evolution is the B200 step in WL mode: a state's canonical_hash is its WL hash, and with
// explore_from_canonical_states_only each WL class is expanded once at its shortest depth.
// Errors throw std::length_error (rule limits, as RuleBuilder does) or std::runtime_error
// (everything else, with the library's message).
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../hgx.h"

namespace hgx {
namespace compat {

namespace detail {

inline void check(hgx_status s) {
    if (s != HGX_OK) throw std::runtime_error(std::string("hgx: ") + hgx_last_error());
}

inline std::vector<uint32_t> rule_blob(const std::vector<std::vector<uint8_t>>& lhs,
                                       const std::vector<std::vector<uint8_t>>& rhs) {
    std::vector<uint32_t> b;
    for (const auto* side : {&lhs, &rhs}) {
        b.push_back(static_cast<uint32_t>(side->size()));
        for (const auto& e : *side) {
            b.push_back(static_cast<uint32_t>(e.size()));
            for (uint8_t v : e) b.push_back(v);
        }
    }
    return b;
}

template <class V>
std::vector<uint32_t> roots_blob(const std::vector<std::vector<std::vector<V>>>& roots) {
    std::vector<uint32_t> b{static_cast<uint32_t>(roots.size())};
    for (const auto& st : roots) {
        b.push_back(static_cast<uint32_t>(st.size()));
        for (const auto& e : st) {
            b.push_back(static_cast<uint32_t>(e.size()));
            for (auto v : e) b.push_back(static_cast<uint32_t>(v));
        }
    }
    return b;
}

struct ResultDeleter {
    void operator()(hgx_result* r) const { hgx_result_free(r); }
};
using ResultPtr = std::shared_ptr<hgx_result>;

struct EngineDeleter {
    void operator()(hgx_engine* e) const { hgx_engine_destroy(e); }
};

template <class T>
std::vector<T> copy_array(const hgx_result* r, hgx_array what) {
    const void* p = nullptr;
    uint64_t n = 0;
    check(hgx_result_view(r, what, &p, &n));
    const T* t = static_cast<const T*>(p);
    return std::vector<T>(t, t + n);
}

}  // namespace detail

// =============================================================================================
// The CPU-engine surface (namespace hypergraph in the reference)
// =============================================================================================
namespace engine {

using VertexId = uint32_t;
using EdgeId = uint32_t;
using StateId = uint32_t;
using EventId = uint32_t;
constexpr uint8_t MAX_ARITY = 16, MAX_PATTERN_EDGES = 16, MAX_VARS = 32;

struct RewriteRule {
    uint16_t index = 0;
    std::vector<std::vector<uint8_t>> lhs, rhs;
    uint8_t num_lhs_edges() const { return static_cast<uint8_t>(lhs.size()); }
    uint8_t num_rhs_edges() const { return static_cast<uint8_t>(rhs.size()); }
};

class RuleBuilder {
    RewriteRule r_;
    template <class C>
    static std::vector<uint8_t> edge(const C& vars, const char* what) {
        if (vars.size() > MAX_ARITY)
            throw std::length_error(std::string("RuleBuilder::") + what + ": edge arity exceeds MAX_ARITY");
        std::vector<uint8_t> e;
        for (auto v : vars) {
            if (static_cast<uint64_t>(v) >= MAX_VARS)
                throw std::length_error(std::string("RuleBuilder::") + what +
                                        ": pattern variable index exceeds MAX_VARS");
            e.push_back(static_cast<uint8_t>(v));
        }
        return e;
    }

public:
    RuleBuilder() = default;
    explicit RuleBuilder(uint16_t index) { r_.index = index; }
    template <class C>
    RuleBuilder& lhs(const C& vars) {
        if (r_.lhs.size() >= MAX_PATTERN_EDGES) throw std::length_error("RuleBuilder::lhs: exceeds MAX_PATTERN_EDGES");
        r_.lhs.push_back(edge(vars, "lhs"));
        return *this;
    }
    RuleBuilder& lhs(std::initializer_list<uint8_t> vars) { return lhs(std::vector<uint8_t>(vars)); }
    template <class C>
    RuleBuilder& rhs(const C& vars) {
        if (r_.rhs.size() >= MAX_PATTERN_EDGES) throw std::length_error("RuleBuilder::rhs: exceeds MAX_PATTERN_EDGES");
        r_.rhs.push_back(edge(vars, "rhs"));
        return *this;
    }
    RuleBuilder& rhs(std::initializer_list<uint8_t> vars) { return rhs(std::vector<uint8_t>(vars)); }
    RewriteRule build() const { return r_; }
};

inline RuleBuilder make_rule(uint16_t index = 0) { return RuleBuilder(index); }

struct CausalEdge {
    EventId producer, consumer;
    EdgeId edge;
};
struct BranchialEdge {
    EventId event1, event2;
};

class CausalGraph {
    detail::ResultPtr r_;

public:
    explicit CausalGraph(detail::ResultPtr r) : r_(std::move(r)) {}
    std::vector<CausalEdge> get_causal_edges() const {
        std::vector<CausalEdge> out;
        if (!r_) return out;
        auto t = detail::copy_array<uint32_t>(r_.get(), HGX_ARR_CAUSAL);
        for (size_t i = 0; i + 2 < t.size(); i += 3) out.push_back({t[i], t[i + 1], t[i + 2]});
        return out;
    }
    std::vector<BranchialEdge> get_branchial_edges() const {
        std::vector<BranchialEdge> out;
        if (!r_) return out;
        auto t = detail::copy_array<uint32_t>(r_.get(), HGX_ARR_BRANCHIAL);
        for (size_t i = 0; i + 1 < t.size(); i += 2) out.push_back({t[i], t[i + 1]});
        return out;
    }
    size_t num_causal_edges() const { return r_ ? hgx_result_count(r_.get(), HGX_COUNT_CAUSAL) : 0; }
    size_t num_branchial_edges() const { return r_ ? hgx_result_count(r_.get(), HGX_COUNT_BRANCHIAL) : 0; }
};

class Hypergraph {
    detail::ResultPtr r_;
    uint8_t event_keys_ = 0;
    friend class ParallelEvolutionEngine;

public:
    // Event canonicalisation (hypergraph.hpp:778): EventSignatureKeys bits over the WL hashes --
    // 1 input state, 2 output state, 4 step, 8 rule (3 = Full). The edge-rank keys need an exact
    // canonical labelling and are rejected.
    void set_event_signature_keys(uint8_t keys) {
        if (keys & ~0xFu) throw std::invalid_argument("event signature keys: edge ranks are not provided");
        event_keys_ = keys;
    }
    uint8_t event_signature_keys() const { return event_keys_; }
    // Raw states: every root plus one per event (hypergraph.hpp:567).
    uint32_t num_states() const { return r_ ? static_cast<uint32_t>(hgx_result_count(r_.get(), HGX_COUNT_RAW_STATES)) : 0; }
    // Canonical events when event canonicalisation is on (hypergraph.cpp:1639-1644).
    uint32_t num_events() const {
        if (!r_) return 0;
        return static_cast<uint32_t>(hgx_result_count(r_.get(), event_keys_ ? HGX_COUNT_CANONICAL_EVENTS : HGX_COUNT_EVENTS));
    }
    uint32_t num_raw_events() const { return r_ ? static_cast<uint32_t>(hgx_result_count(r_.get(), HGX_COUNT_EVENTS)) : 0; }
    // Distinct WL canonical hashes.
    size_t num_canonical_states() const { return r_ ? hgx_result_count(r_.get(), HGX_COUNT_CLASSES) : 0; }
    // The recorded states' WL hashes (every raw state in full multiway, one per class in quotient).
    std::vector<uint64_t> canonical_hashes() const {
        return r_ ? detail::copy_array<uint64_t>(r_.get(), HGX_ARR_STATE_HASH) : std::vector<uint64_t>{};
    }
    CausalGraph causal_graph() const { return CausalGraph(r_); }
    const hgx_result* result() const { return r_.get(); }
};

class ParallelEvolutionEngine {
public:
    enum class ExecutionMode { Parallel, Serial };   // accepted for signature compatibility
    explicit ParallelEvolutionEngine(Hypergraph* hg, size_t num_threads = 0,
                                     ExecutionMode mode = ExecutionMode::Parallel, int device = 0)
        : hg_(hg) {
        (void)num_threads;
        (void)mode;
        hgx_engine* e = nullptr;
        detail::check(hgx_engine_create(device, &e));
        eng_.reset(e, detail::EngineDeleter());
    }
    void add_rule(const RewriteRule& r) {
        auto b = detail::rule_blob(r.lhs, r.rhs);
        detail::check(hgx_engine_add_rule(eng_.get(), b.data(), b.size()));
    }
    void set_transitive_reduction(bool enable) {
        detail::check(hgx_engine_set_option(eng_.get(), HGX_OPT_TRANSITIVE_REDUCTION, enable ? 1 : 0));
    }
    void set_explore_from_canonical_states_only(bool enable) {
        detail::check(hgx_engine_set_option(eng_.get(), HGX_OPT_QUOTIENT, enable ? 1 : 0));
    }
    void set_max_states(size_t n) { detail::check(hgx_engine_set_option(eng_.get(), HGX_OPT_MAX_STATES, n)); }
    void evolve(const std::vector<std::vector<VertexId>>& initial_edges, size_t steps) {
        run(detail::roots_blob(std::vector<std::vector<std::vector<VertexId>>>{initial_edges}), steps);
    }
    void evolve(const std::vector<std::vector<std::vector<VertexId>>>& initial_states, size_t steps) {
        run(detail::roots_blob(initial_states), steps);
    }
    size_t num_states() const { return hg_->num_states(); }
    size_t num_canonical_states() const { return hg_->num_canonical_states(); }
    size_t num_events() const { return hg_->num_events(); }
    size_t num_causal_edges() const { return hg_->causal_graph().num_causal_edges(); }
    size_t num_branchial_edges() const { return hg_->causal_graph().num_branchial_edges(); }

private:
    void run(const std::vector<uint32_t>& blob, size_t steps) {
        detail::check(hgx_engine_set_option(eng_.get(), HGX_OPT_EVENT_SIGNATURE_KEYS, hg_->event_keys_));
        hgx_result* r = nullptr;
        detail::check(hgx_evolve(eng_.get(), blob.data(), blob.size(), static_cast<uint32_t>(steps), &r));
        hg_->r_.reset(r, detail::ResultDeleter());
    }
    Hypergraph* hg_;
    std::shared_ptr<hgx_engine> eng_;
};

}  // namespace engine

}  // namespace compat
}  // namespace hgx

// The GPU-engine surface (hg_gpu::evolve, Engine, PersistentEvolver and their DTOs).
#include "hg_gpu.hpp"
