// hgx/hg_gpu.hpp -- the reference's GPU-engine surface (gpu/include/hg_gpu/evolve.hpp), header
// only, over the C ABI (hgx.h).
//
// A drop-in for code written against hg_gpu::evolve / Engine / PersistentEvolver: the same DTO
// names, fields, defaults and error behaviour (capacity problems become `warnings` on a partial
// result; invalid inputs throw std::invalid_argument; driver failures throw std::runtime_error).
// The evolution is the B200 multiway step in WL mode:
//
//   * a state's canonical_hash is its WL hash (the reference's shared WL core); exact IR
//     canonicalisation is not computed on this path, so CanonicalizationMode::Full is served by
//     WL classes (they coincide with IR classes except on rare WL collisions);
//   * explore_from_canonical_states_only with canonicalization Full expands each WL class once,
//     at its shortest depth; with canonicalization None every state is its own class, i.e. full
//     multiway;
//   * the sampling and capping options of the reference (exploration_probability,
//     transition_rate, rule_weights, max_states_per_step, max_successor_states_per_parent,
//     matches_per_state_rule) and Automatic event identity are rejected when set; sessions
//     (run with a SessionView) are refused, as the reference refuses a steered session.
//
// Types live in hgx::compat::gpu. The reference spells them hg_gpu::...; this header makes that
// name resolve here: if the reference's namespace root (HG_NAMESPACE, from hgcommon/namespace.hpp)
// is already declared, these types are made visible inside HG_NAMESPACE::gpu, which the
// reference's own `hg_gpu` alias names; otherwise `hg_gpu` is declared as an alias of
// hgx::compat::gpu. Define HGX_NO_HG_GPU_ALIAS to skip both.
#pragma once
#include <algorithm>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "compat.hpp"

namespace hgx {
namespace compat {
namespace gpu {

using VertexId = uint32_t;
using StateId = uint32_t;
using EventId = uint32_t;
using EdgeId = uint32_t;
using RuleId = uint32_t;
constexpr uint32_t INVALID_ID = 0xFFFFFFFFu;
constexpr uint32_t MAX_VARS = 32;

// gpu/include/hg_gpu/types.hpp:118-128 (the two enums have different orders there too).
enum class CanonicalizationMode : uint8_t { None = 0, Automatic, Full };
enum class EventCanonicalizationMode : uint8_t { None = 0, Full, Automatic };

// common/include/hgcommon/core.hpp:128-155: which artifacts a run records.
struct RecordSet {
    bool causal = true;
    bool branchial = true;
    bool state_events = true;
    bool raw_events = true;
};

// gpu/include/hg_gpu/overflow.hpp: the capacity kinds this path can report.
enum class ErrorKind : uint32_t {
    kStatePoolFull = 3,       // the state cap stopped the evolution
    kDeviceOutOfMemory = 21,  // max_device_memory_bytes (or the device) ran out
    kCount = 32
};

inline const char* error_kind_name(ErrorKind k) {
    switch (k) {
        case ErrorKind::kStatePoolFull: return "StatePoolFull";
        case ErrorKind::kDeviceOutOfMemory: return "DeviceOutOfMemory";
        default: return "Unknown";
    }
}

struct OverflowWarning {
    ErrorKind kind;
    uint32_t count;
    std::string context;
};

struct RewriteRule {
    std::vector<std::vector<uint8_t>> lhs;
    std::vector<std::vector<uint8_t>> rhs;
    uint8_t num_lhs_vars = 0;
    uint8_t num_rhs_vars = 0;
};

// gpu/include/hg_gpu/evolve.hpp:27-142, field for field, plus max_states (a cap on the states
// recorded: WL classes under quotient exploration, raw states otherwise; 0 = unlimited).
struct EvolveInput {
    RecordSet record;
    bool edge_identity = false;
    std::vector<RewriteRule> rules;
    std::vector<std::vector<VertexId>> initial_state;
    std::vector<std::vector<std::vector<VertexId>>> initial_states;   // takes precedence
    bool quotient_initial_states = false;
    uint32_t num_steps = 0;
    CanonicalizationMode canonicalization = CanonicalizationMode::Full;
    EventCanonicalizationMode event_canonicalization = EventCanonicalizationMode::None;
    bool transitive_reduction = true;
    // Relations are always materialised on this path (there is no quotient reconstruction).
    bool materialize_relations = false;
    bool explore_from_canonical_states_only = true;
    float exploration_probability = 1.0f;
    uint64_t exploration_seed = 0;
    double transition_rate = 1.0;
    std::vector<double> rule_weights;
    uint32_t max_states_per_step = 0;
    uint32_t max_successor_states_per_parent = 0;
    uint32_t matches_per_state_rule = 0;
    // Sizing overrides of the reference's fixed pools; this engine grows its arrays on demand.
    uint32_t slice_scan_max_edges = 0;
    uint32_t max_blocks_per_launch = 0;
    // 0 resolves to 90% of the device's memory, as in the reference.
    uint64_t max_device_memory_bytes = 0;
    uint64_t max_states = 0;
};

struct CanonicalState {
    StateId id = INVALID_ID;
    uint64_t canonical_hash = 0;
    std::vector<std::vector<VertexId>> edges;
};

struct Event {
    EventId id = INVALID_ID;
    EventId canonical_id = INVALID_ID;   // first event with the same signature (itself when off)
    uint64_t signature = 0;              // 0 under EventCanonicalizationMode::None
    StateId input_state = INVALID_ID;
    StateId output_state = INVALID_ID;
    RuleId rule = 0;
    uint32_t step = 0;
    std::vector<EdgeId> consumed_edges;
    std::vector<EdgeId> produced_edges;
};

struct CausalEdge {
    EventId from;
    EventId to;
};

struct BranchialEdge {
    EventId a;
    EventId b;
};

struct EvolveResult {
    std::vector<CanonicalState> states;
    // With edge_identity: each state's global edge ids, and edge id -> vertices for every edge of
    // a recorded state (every edge in full multiway; under quotient exploration the edges of the
    // class representatives -- an edge minted by an event whose child was a duplicate is held by
    // no recorded state and has an empty entry).
    std::vector<std::vector<EdgeId>> state_edge_ids;
    std::vector<std::vector<VertexId>> global_edges;
    std::vector<Event> events;
    std::vector<CausalEdge> causal_edges;       // one per (producer, consumer, edge) triple
    std::vector<BranchialEdge> branchial_edges;
    std::vector<OverflowWarning> warnings;
    // The quotient-reconstruction fields of the reference: this path records the explored
    // relations directly, so the reconstruction never runs and these stay zero / empty.
    uint32_t expansion_matches = 0;
    uint32_t expansion_instances = 0;
    uint32_t reconstructed_raw_events = 0;
    bool reconstruction_ran = false;
    uint32_t reconstructed_events = 0;
    uint32_t reconstructed_causal_pairs = 0;
    uint32_t reconstructed_causal_edges = 0;
    uint32_t reconstructed_causal_pairs_reduced = 0;
    uint32_t reconstructed_branchial = 0;
    std::vector<std::pair<uint64_t, uint64_t>> reconstructed_causal_relation;
    std::vector<std::pair<uint64_t, uint64_t>> reconstructed_causal_relation_reduced;
    std::vector<std::pair<uint64_t, uint64_t>> reconstructed_branchial_relation;
    std::vector<uint64_t> reconstructed_event_signature;
    uint32_t frame_alignments = 0;
    uint32_t frame_align_failures = 0;
    // Distinct WL classes among the recorded states (no reference counterpart).
    uint64_t num_classes = 0;

    // Events a caller is told: the canonical events (each its own canonical) -- the raw count
    // under EventCanonicalizationMode::None.
    size_t observable_num_events() const {
        size_t n = 0;
        for (const auto& e : events) n += (e.canonical_id == e.id || e.canonical_id == INVALID_ID) ? 1 : 0;
        return n;
    }
    // Causal (producer, consumer) pairs, deduplicated as the FFI reports them. The relation is
    // already reduced when transitive_reduction was on, so `reduced` selects nothing further.
    size_t observable_num_causal_pairs(bool reduced) const {
        (void)reduced;
        std::vector<uint64_t> k;
        k.reserve(causal_edges.size());
        for (const auto& c : causal_edges) k.push_back((uint64_t(c.from) << 32) | c.to);
        std::sort(k.begin(), k.end());
        return static_cast<size_t>(std::unique(k.begin(), k.end()) - k.begin());
    }
    size_t observable_num_branchial() const { return branchial_edges.size(); }
};

// gpu/include/hg_gpu/evolve.hpp:176-320. The reference sizes fixed device pools from these and
// grows them by retrying on overflow; this engine grows its arrays on demand, so the fields are
// the sizes a run is expected to reach (they feed estimated_device_bytes), and `device` picks
// the GPU.
struct EngineConfig {
    uint32_t max_edges = 1u << 16;
    uint32_t max_vertices = 1u << 16;
    uint32_t max_vertex_slots = 1u << 18;
    uint32_t max_states = 1u << 14;
    uint32_t max_state_edge_total = 1u << 22;
    uint32_t sig_index_buckets = 1024;
    uint32_t inverted_pool = 1u << 18;
    uint32_t sig_index_pool = 1u << 16;
    uint32_t canonical_map_slots = 1u << 14;
    uint32_t match_dedup_slots = 1u << 16;
    uint32_t slice_scan_max_edges = 256;
    uint32_t max_blocks_per_launch = 0;
    uint32_t event_canon_slots = 1u << 16;
    uint32_t reconstruction_max_depth = 0;
    uint32_t max_events = 1u << 16;
    uint32_t max_causal_edges = 1u << 18;
    uint32_t max_branchial_edges = 1u << 18;
    uint32_t causal_triple_slots = 1u << 19;
    uint32_t causal_pair_slots = 1u << 18;
    uint32_t branchial_pair_slots = 1u << 19;
    uint32_t edge_consumer_nodes = 1u << 18;
    uint32_t branchial_index_buckets = 1u << 16;
    uint32_t branchial_index_nodes = 1u << 18;
    uint32_t tr_preds_nodes = 1u << 20;
    uint32_t qe_capacity_scale = 1u;
    uint32_t ir_arena_share_words = 65536;
    uint32_t ir_generators = 32;
    uint32_t ir_depth = 8;
    int device = 0;
};

namespace detail {

inline hgx_job job_view(const std::vector<uint32_t>& rules, const std::vector<uint32_t>& roots,
                        uint32_t steps, bool quotient, uint64_t max_states) {
    hgx_job j;
    j.rules = rules.data();
    j.rules_len = rules.size();
    j.roots = roots.data();
    j.roots_len = roots.size();
    j.steps = steps;
    j.quotient = quotient ? 1u : 0u;
    j.max_states = max_states;
    return j;
}

inline std::vector<uint32_t> rules_blob(const std::vector<RewriteRule>& rules) {
    std::vector<uint32_t> b{static_cast<uint32_t>(rules.size())};
    for (const auto& r : rules) {
        auto one = compat::detail::rule_blob(r.lhs, r.rhs);
        b.insert(b.end(), one.begin(), one.end());
    }
    return b;
}

inline std::vector<std::vector<std::vector<VertexId>>> roots_of(const EvolveInput& in) {
    if (!in.initial_states.empty()) return in.initial_states;
    return {in.initial_state};
}

// The options this path does not provide, rejected rather than silently ignored.
inline void validate(const EvolveInput& in) {
    if (in.rules.empty()) throw std::invalid_argument("evolve: no rules");
    for (const auto& r : in.rules)
        if (r.lhs.empty()) throw std::invalid_argument("evolve: a rule has an empty left-hand side");
    if (in.exploration_probability != 1.0f || in.transition_rate != 1.0 ||
        in.max_states_per_step || in.max_successor_states_per_parent || in.matches_per_state_rule)
        throw std::invalid_argument("evolve: sampling and per-step capping options are not provided "
                                    "on this path (exploration_probability, transition_rate, "
                                    "max_states_per_step, max_successor_states_per_parent, "
                                    "matches_per_state_rule must keep their defaults)");
    for (double w : in.rule_weights)
        if (w != 1.0) throw std::invalid_argument("evolve: rule_weights other than 1 are not provided");
    if (in.event_canonicalization == EventCanonicalizationMode::Automatic)
        throw std::invalid_argument("evolve: Automatic event identity needs exact edge ranks, which "
                                    "this path does not compute (use Full or None)");
    if (in.canonicalization == CanonicalizationMode::Automatic && in.explore_from_canonical_states_only)
        throw std::invalid_argument("evolve: content-keyed (Automatic) quotient exploration is not "
                                    "provided; use Full (WL classes) or explore every state");
}

inline bool quotient_of(const EvolveInput& in) {
    return in.explore_from_canonical_states_only && in.canonicalization == CanonicalizationMode::Full;
}

inline uint64_t device_limit(const EvolveInput& in, int device) {
    if (in.max_device_memory_bytes) return in.max_device_memory_bytes;
    uint64_t f = 0, t = 0;
    if (hgx_device_memory(device, &f, &t) != HGX_OK) return 0;
    return t / 10 * 9;
}

inline EvolveResult convert(const hgx_result* rr, const EvolveInput& in) {
    using compat::detail::copy_array;
    EvolveResult out;
    auto hash = copy_array<uint64_t>(rr, HGX_ARR_STATE_HASH);
    auto eoff = copy_array<uint32_t>(rr, HGX_ARR_STATE_EDGE_OFF);
    auto eids = copy_array<uint32_t>(rr, HGX_ARR_STATE_EDGE_IDS);
    auto ar = copy_array<uint8_t>(rr, HGX_ARR_STATE_ARITY);
    auto voff = copy_array<uint32_t>(rr, HGX_ARR_STATE_VERT_OFF);
    auto verts = copy_array<uint32_t>(rr, HGX_ARR_STATE_VERTS);
    out.states.resize(hash.size());
    if (in.edge_identity) out.state_edge_ids.resize(hash.size());
    for (size_t s = 0; s < hash.size(); ++s) {
        out.states[s].id = static_cast<StateId>(s);
        out.states[s].canonical_hash = hash[s];
        if (eoff.size() > s + 1) {
            uint32_t v = voff[s];
            for (uint32_t k = eoff[s]; k < eoff[s + 1]; ++k) {
                out.states[s].edges.emplace_back(verts.begin() + v, verts.begin() + v + ar[k]);
                if (in.edge_identity) {
                    const uint32_t id = eids[k];
                    if (out.global_edges.size() <= id) out.global_edges.resize(id + 1);
                    if (out.global_edges[id].empty())
                        out.global_edges[id].assign(verts.begin() + v, verts.begin() + v + ar[k]);
                }
                v += ar[k];
            }
            if (in.edge_identity)
                out.state_edge_ids[s].assign(eids.begin() + eoff[s], eids.begin() + eoff[s + 1]);
        }
    }
    if (in.record.raw_events) {
        auto ev = copy_array<uint32_t>(rr, HGX_ARR_EVENTS);
        auto coff = copy_array<uint32_t>(rr, HGX_ARR_EVENT_CONS_OFF);
        auto cons = copy_array<uint32_t>(rr, HGX_ARR_EVENT_CONS);
        auto prod = copy_array<uint32_t>(rr, HGX_ARR_EVENT_PROD);
        auto sig = copy_array<uint64_t>(rr, HGX_ARR_EVENT_SIG);
        std::unordered_map<uint64_t, EventId> first_of;
        out.events.resize(ev.size() / 4);
        for (size_t i = 0; i < out.events.size(); ++i) {
            Event& x = out.events[i];
            x.id = static_cast<EventId>(i);
            x.canonical_id = x.id;
            if (sig.size() == out.events.size()) {
                x.signature = sig[i];
                x.canonical_id = first_of.emplace(sig[i], x.id).first->second;
            }
            x.input_state = ev[4 * i];
            x.output_state = ev[4 * i + 1];
            x.rule = ev[4 * i + 2];
            x.step = ev[4 * i + 3];
            x.consumed_edges.assign(cons.begin() + coff[i], cons.begin() + coff[i + 1]);
            for (uint32_t k = 0; k < prod[2 * i + 1]; ++k) x.produced_edges.push_back(prod[2 * i] + k);
        }
    }
    auto ca = copy_array<uint32_t>(rr, HGX_ARR_CAUSAL);
    for (size_t i = 0; i + 2 < ca.size(); i += 3) out.causal_edges.push_back({ca[i], ca[i + 1]});
    auto br = copy_array<uint32_t>(rr, HGX_ARR_BRANCHIAL);
    for (size_t i = 0; i + 1 < br.size(); i += 2) out.branchial_edges.push_back({br[i], br[i + 1]});
    out.num_classes = hgx_result_count(rr, HGX_COUNT_CLASSES);
    if (hgx_result_count(rr, HGX_COUNT_TRUNCATED))
        out.warnings.push_back({ErrorKind::kStatePoolFull, 1u,
                                "state cap: the evolution stopped at max_states"});
    return out;
}

}  // namespace detail

// Sizes a run of `input` is expected to reach (gpu/include/hg_gpu/evolve.hpp:404).
inline EngineConfig config_from_input(const EvolveInput& input) {
    EngineConfig cfg;
    auto roots = detail::roots_of(input);
    const auto rules = detail::rules_blob(input.rules);
    const auto blob = compat::detail::roots_blob(roots);
    const hgx_job job = detail::job_view(rules, blob, input.num_steps, detail::quotient_of(input),
                                         input.max_states);
    uint64_t bytes = 0;
    compat::detail::check(hgx_estimate_device_bytes(&job, &bytes));
    // the estimate's own per-state figure is ~1-2 KB: express it back as state / event counts
    const uint64_t states = std::max<uint64_t>(1u << 14, std::min<uint64_t>(bytes / 2048, 1ull << 31));
    cfg.max_states = static_cast<uint32_t>(states);
    cfg.canonical_map_slots = static_cast<uint32_t>(std::min<uint64_t>(4 * states, 1ull << 31));
    cfg.max_events = static_cast<uint32_t>(std::min<uint64_t>(8 * states, 0xFFFFFFFFull));
    cfg.max_edges = static_cast<uint32_t>(std::min<uint64_t>(16 * states, 0xFFFFFFFFull));
    cfg.reconstruction_max_depth = input.num_steps;
    return cfg;
}

// Conservative device bytes of an engine of this size (gpu/include/hg_gpu/evolve.hpp:409);
// monotonic in every capacity field.
inline uint64_t estimated_device_bytes(const EngineConfig& cfg) {
    const uint64_t per_state = 56 + 48 + 4ull * 40;
    const uint64_t per_event = 112 + 32 + 128;
    return uint64_t(cfg.max_states) * per_state + uint64_t(cfg.max_events) * per_event +
           uint64_t(cfg.max_edges) * 4 + uint64_t(cfg.canonical_map_slots) * 12 +
           uint64_t(cfg.max_causal_edges) * 12 + uint64_t(cfg.max_branchial_edges) * 8 + (1ull << 20);
}

// gpu/include/hg_gpu/evolve.hpp:389-400: an opaque session handle. Sessions (continuing an
// evolution across calls) are not provided on this path; a run given one refuses.
struct SessionView;

class GpuSession {
public:
    GpuSession(uint32_t max_states, uint32_t max_events) : states_(max_states), events_(max_events) {}
    GpuSession(const GpuSession&) = delete;
    GpuSession& operator=(const GpuSession&) = delete;
    SessionView* view() { return reinterpret_cast<SessionView*>(this); }
    uint32_t frontier_size() const { return 0; }

private:
    uint32_t states_, events_;
};

// gpu/include/hg_gpu/evolve.hpp:435-455: device state that runs many inputs back to back.
class Engine {
public:
    explicit Engine(EngineConfig cfg) : cfg_(cfg) {
        hgx_engine* e = nullptr;
        compat::detail::check(hgx_engine_create(cfg.device, &e));
        eng_.reset(e, compat::detail::EngineDeleter());
    }
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Capacity overflows (the state cap, the device-memory ceiling) become `warnings` on a
    // partial result; invalid inputs throw std::invalid_argument.
    EvolveResult run(const EvolveInput& input, SessionView* session = nullptr, uint32_t start_step = 0) {
        if (session || start_step)
            throw std::invalid_argument("Engine::run: sessions (continuing an evolution across calls) "
                                        "are not provided on this path");
        detail::validate(input);
        hgx_engine* e = eng_.get();
        compat::detail::check(hgx_engine_clear_rules(e));
        for (const auto& r : input.rules) {
            auto b = compat::detail::rule_blob(r.lhs, r.rhs);
            compat::detail::check(hgx_engine_add_rule(e, b.data(), b.size()));
        }
        const bool quotient = detail::quotient_of(input);
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_TRANSITIVE_REDUCTION, input.transitive_reduction));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_QUOTIENT, quotient));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_KEEP_STATE_EDGES, 1));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_KEEP_STATE_EDGE_IDS, input.edge_identity));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_MAX_STATES, input.max_states));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_RECORD_CAUSAL, input.record.causal));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_RECORD_BRANCHIAL, input.record.branchial));
        compat::detail::check(hgx_engine_set_option(
            e, HGX_OPT_EVENT_SIGNATURE_KEYS,
            input.event_canonicalization == EventCanonicalizationMode::Full ? 3 : 0));
        compat::detail::check(hgx_engine_set_option(e, HGX_OPT_MAX_DEVICE_BYTES,
                                                    detail::device_limit(input, cfg_.device)));
        auto roots = detail::roots_of(input);
        if (input.quotient_initial_states && quotient && roots.size() > 1) roots = distinct_roots(roots);
        const auto blob = compat::detail::roots_blob(roots);
        hgx_result* rr = nullptr;
        const hgx_status st = hgx_evolve(e, blob.data(), blob.size(), input.num_steps, &rr);
        if (st == HGX_ERR_CAPACITY) {
            EvolveResult out;
            out.warnings.push_back({ErrorKind::kDeviceOutOfMemory, 1u, hgx_last_error()});
            return out;
        }
        compat::detail::check(st);
        std::unique_ptr<hgx_result, compat::detail::ResultDeleter> res(rr);
        return detail::convert(rr, input);
    }
    void reset() {}   // every run starts from an empty engine (its allocations are kept)
    const EngineConfig& config() const { return cfg_; }
    hgx_engine* handle() const { return eng_.get(); }

private:
    // Isomorphic roots collapse to one under quotient_initial_states (evolve.hpp:46-49): roots
    // with equal WL hashes keep the first.
    std::vector<std::vector<std::vector<VertexId>>> distinct_roots(
        const std::vector<std::vector<std::vector<VertexId>>>& roots) {
        hgx_engine* e = eng_.get();
        const auto blob = compat::detail::roots_blob(roots);
        hgx_result* rr = nullptr;
        compat::detail::check(hgx_evolve(e, blob.data(), blob.size(), 0, &rr));
        std::unique_ptr<hgx_result, compat::detail::ResultDeleter> res(rr);
        auto hash = compat::detail::copy_array<uint64_t>(rr, HGX_ARR_STATE_HASH);
        std::vector<std::vector<std::vector<VertexId>>> out;
        std::vector<uint64_t> seen;
        for (size_t i = 0; i < roots.size() && i < hash.size(); ++i) {
            if (std::find(seen.begin(), seen.end(), hash[i]) != seen.end()) continue;
            seen.push_back(hash[i]);
            out.push_back(roots[i]);
        }
        return out;
    }

    EngineConfig cfg_;
    std::shared_ptr<hgx_engine> eng_;
};

// gpu/include/hg_gpu/evolve.hpp:368: one-shot evolve on a fresh engine.
inline EvolveResult evolve(const EvolveInput& input) {
    Engine engine(config_from_input(input));
    return engine.run(input);
}

// gpu/include/hg_gpu/evolve.hpp:464-497: one engine kept across runs (its device arrays are
// reused; the engine grows on demand and never shrinks).
class PersistentEvolver {
public:
    PersistentEvolver() = default;
    PersistentEvolver(const PersistentEvolver&) = delete;
    PersistentEvolver& operator=(const PersistentEvolver&) = delete;

    EvolveResult run(const EvolveInput& input) {
        if (!engine_) {
            cfg_ = config_from_input(input);
            engine_ = std::make_unique<Engine>(cfg_);
        }
        return engine_->run(input);
    }

    struct SessionRun {
        EvolveResult result;
        bool ok = false;
        std::string error;
    };
    SessionRun run_session(const EvolveInput& input, SessionView* session, uint32_t start_step) {
        (void)input;
        (void)session;
        (void)start_step;
        SessionRun r;
        r.error = "sessions (continuing an evolution across calls) are not provided on this path";
        return r;
    }

    bool has_engine() const { return engine_ != nullptr; }
    const EngineConfig& engine_config() const { return cfg_; }

private:
    std::unique_ptr<Engine> engine_;
    EngineConfig cfg_{};
};

}  // namespace gpu
}  // namespace compat
}  // namespace hgx

#ifndef HGX_NO_HG_GPU_ALIAS
#ifdef HG_NAMESPACE
namespace HG_NAMESPACE {
namespace gpu {
using namespace ::hgx::compat::gpu;
}  // namespace gpu
}  // namespace HG_NAMESPACE
#else
namespace hg_gpu = ::hgx::compat::gpu;
#endif
#endif
