// extern "C" boundary of the multiway step (declared in include/hgx.h).
#include "../../include/hgx.h"

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"

struct hgx_engine {
    hgx::Engine engine;
    std::vector<hgx::RuleSpec> rules;
    bool quotient = false;
    uint64_t max_states = 0;
    hgx::RunOptions opt;
    explicit hgx_engine(int dev) : engine(dev) {}
};

struct hgx_result {
    hgx::EvolutionResult r;
    std::vector<uint32_t> events_flat;   // (in, out, rule, step) for vector-held results
    std::vector<uint32_t> prod_flat;     // (first, count)
    const void* ptr[hgx::ResultArrays::kArrays] = {};   // every array, indexed by hgx_array
    uint64_t count[hgx::ResultArrays::kArrays] = {};    // elements
};

namespace {

thread_local std::string g_err;

hgx_status fail(hgx_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

template <class F>
hgx_status guarded(F&& f) {
    try {
        g_err.clear();
        return f();
    } catch (const hgx::CudaError& e) {
        return fail(HGX_ERR_CUDA, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(HGX_ERR_INVALID, e.what());
    } catch (const std::length_error& e) {
        return fail(HGX_ERR_INVALID, e.what());
    } catch (const std::exception& e) {
        const std::string m = e.what();
        if (m.find("no CUDA device") != std::string::npos) return fail(HGX_ERR_NO_DEVICE, m);
        if (m.find("capacity") != std::string::npos || m.find("exhausted") != std::string::npos)
            return fail(HGX_ERR_CAPACITY, m);
        return fail(HGX_ERR_INTERNAL, m);
    } catch (...) {
        return fail(HGX_ERR_INTERNAL, "unknown error");
    }
}

struct Reader {
    const uint32_t* p;
    size_t n, i = 0;
    uint32_t get() {
        if (i >= n) throw std::invalid_argument("blob: truncated");
        return p[i++];
    }
};

std::vector<std::vector<uint8_t>> read_pattern_edges(Reader& r) {
    const uint32_t ne = r.get();
    if (ne > 16) throw std::length_error("rule: more than 16 pattern edges (MAX_PATTERN_EDGES)");
    std::vector<std::vector<uint8_t>> out(ne);
    for (auto& e : out) {
        const uint32_t a = r.get();
        if (a == 0 || a > 16) throw std::length_error("rule: edge arity must be 1..16 (MAX_ARITY)");
        e.resize(a);
        for (auto& v : e) {
            const uint32_t x = r.get();
            if (x >= 32) throw std::length_error("rule: pattern variable index exceeds MAX_VARS");
            v = static_cast<uint8_t>(x);
        }
    }
    return out;
}

hgx::RuleSpec read_rule(Reader& r) {
    hgx::RuleSpec s;
    s.lhs = read_pattern_edges(r);
    s.rhs = read_pattern_edges(r);
    if (s.lhs.empty()) throw std::invalid_argument("rule: empty left-hand side");
    return s;
}

std::vector<hgx::RuleSpec> read_rules(const uint32_t* p, size_t n) {
    Reader r{p, n};
    const uint32_t nr = r.get();
    std::vector<hgx::RuleSpec> out;
    for (uint32_t i = 0; i < nr; ++i) out.push_back(read_rule(r));
    return out;
}

std::vector<std::vector<std::vector<uint32_t>>> read_roots(const uint32_t* p, size_t n) {
    Reader r{p, n};
    const uint32_t nr = r.get();
    std::vector<std::vector<std::vector<uint32_t>>> out(nr);
    for (auto& st : out) {
        const uint32_t ne = r.get();
        st.resize(ne);
        for (auto& e : st) {
            const uint32_t a = r.get();
            if (a == 0 || a > 16) throw std::invalid_argument("state: edge arity must be 1..16");
            e.resize(a);
            for (auto& v : e) v = r.get();
        }
    }
    return out;
}

hgx::EvolutionSpec spec_of(const hgx_job& j) {
    if (!j.rules || !j.roots) throw std::invalid_argument("job: null rules or roots");
    hgx::EvolutionSpec s;
    s.rules = read_rules(j.rules, j.rules_len);
    s.roots = read_roots(j.roots, j.roots_len);
    s.steps = j.steps;
    s.quotient = j.quotient != 0;
    s.max_states = j.max_states;
    return s;
}

hgx_result* wrap(hgx::EvolutionResult&& r) {
    auto* out = new hgx_result;
    out->r = std::move(r);
    auto& x = out->r;
    if (x.flat) {
        for (int i = 0; i < hgx::ResultArrays::kArrays; ++i) {
            out->ptr[i] = x.flat->ptr[i];
            out->count[i] = x.flat->count[i];
        }
        return out;
    }
    out->events_flat.resize(4 * x.ev_in.size());
    out->prod_flat.resize(2 * x.ev_in.size());
    for (size_t i = 0; i < x.ev_in.size(); ++i) {
        out->events_flat[4 * i] = x.ev_in[i];
        out->events_flat[4 * i + 1] = x.ev_out[i];
        out->events_flat[4 * i + 2] = x.ev_rule[i];
        out->events_flat[4 * i + 3] = x.ev_step[i];
        out->prod_flat[2 * i] = x.ev_prod_first[i];
        out->prod_flat[2 * i + 1] = x.ev_prod_count[i];
    }
    if (x.ev_cons_off.empty()) x.ev_cons_off.push_back(0);
    if (x.state_edge_off.empty()) x.state_edge_off.push_back(0);
    if (x.state_vert_off.empty()) x.state_vert_off.push_back(0);
    for (uint32_t ev : x.state_event) x.n_roots += (ev == 0xFFFFFFFFu) ? 1 : 0;
    auto set = [&](int i, const auto& v) {
        out->ptr[i] = v.data();
        out->count[i] = v.size();
    };
    set(HGX_ARR_STATE_HASH, x.state_hash);
    set(HGX_ARR_STATE_DEPTH, x.state_depth);
    set(HGX_ARR_EVENTS, out->events_flat);
    set(HGX_ARR_CAUSAL, x.causal);
    set(HGX_ARR_BRANCHIAL, x.branchial);
    set(HGX_ARR_EVENT_CONS_OFF, x.ev_cons_off);
    set(HGX_ARR_EVENT_CONS, x.ev_cons);
    set(HGX_ARR_EVENT_PROD, out->prod_flat);
    set(HGX_ARR_STATE_EDGE_OFF, x.state_edge_off);
    set(HGX_ARR_STATE_EDGE_IDS, x.state_edge_ids);
    set(HGX_ARR_STATE_ARITY, x.state_arity);
    set(HGX_ARR_STATE_VERT_OFF, x.state_vert_off);
    set(HGX_ARR_STATE_VERTS, x.state_verts);
    set(HGX_ARR_EVENT_SIG, x.ev_sig);
    return out;
}

}  // namespace

void hgx::set_last_error(const std::string& msg) { g_err = msg; }

extern "C" {

const char* hgx_last_error(void) { return g_err.c_str(); }

const char* hgx_version(void) { return "hgx 0.1 (sm_100a)"; }

hgx_status hgx_engine_create(int device, hgx_engine** out) {
    if (!out) return fail(HGX_ERR_INVALID, "null output pointer");
    return guarded([&] {
        *out = new hgx_engine(device);
        return HGX_OK;
    });
}

void hgx_engine_destroy(hgx_engine* e) {
    try {
        delete e;
    } catch (...) {
    }
}

hgx_status hgx_engine_add_rule(hgx_engine* e, const uint32_t* rule, size_t len) {
    if (!e || !rule) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        Reader r{rule, len};
        e->rules.push_back(read_rule(r));
        return HGX_OK;
    });
}

hgx_status hgx_engine_clear_rules(hgx_engine* e) {
    if (!e) return fail(HGX_ERR_INVALID, "null engine");
    e->rules.clear();
    return HGX_OK;
}

hgx_status hgx_engine_set_option(hgx_engine* e, hgx_option opt, uint64_t value) {
    if (!e) return fail(HGX_ERR_INVALID, "null engine");
    switch (opt) {
        case HGX_OPT_QUOTIENT: e->quotient = value != 0; return HGX_OK;
        case HGX_OPT_MAX_STATES: e->max_states = value; return HGX_OK;
        case HGX_OPT_TRANSITIVE_REDUCTION: e->opt.transitive_reduction = value != 0; return HGX_OK;
        case HGX_OPT_RECORD_CAUSAL: e->opt.causal = value != 0; return HGX_OK;
        case HGX_OPT_RECORD_BRANCHIAL: e->opt.branchial = value != 0; return HGX_OK;
        case HGX_OPT_KEEP_STATE_EDGES: e->opt.keep_state_edges = value != 0; return HGX_OK;
        case HGX_OPT_TIMING:
            if (value > 2) return fail(HGX_ERR_INVALID, "timing: 0 off, 1 every stage, 2 the expand kernel only");
            e->engine.set_timing(static_cast<int>(value));
            return HGX_OK;
        case HGX_OPT_READBACK: e->opt.readback = value != 0; return HGX_OK;
        case HGX_OPT_FORWARDING:
            if (value > 2) return fail(HGX_ERR_INVALID, "forwarding mode must be 0, 1 or 2");
            e->opt.forwarding = static_cast<uint32_t>(value);
            return HGX_OK;
        case HGX_OPT_CHUNK_MIN: e->opt.chunk_min = value; return HGX_OK;
        case HGX_OPT_LEVEL_SPLIT: e->opt.level_split = value; return HGX_OK;
        case HGX_OPT_MAX_DEVICE_BYTES: e->engine.set_device_limit(value); return HGX_OK;
        case HGX_OPT_JOIN_INDEX: e->opt.join_index = value != 0; return HGX_OK;
        case HGX_OPT_KEEP_STATE_EDGE_IDS: e->opt.keep_state_edge_ids = value != 0; return HGX_OK;
        case HGX_OPT_STREAM_RESULT:
            if (value > 2) return fail(HGX_ERR_INVALID, "stream result: 0 off, 1 results of 64 MB or more, 2 always");
            e->opt.stream_result = static_cast<uint32_t>(value);
            return HGX_OK;
        case HGX_OPT_LANE_JOIN:
            if (value > 2) return fail(HGX_ERR_INVALID, "lane join must be 0 (autotuned), 1 or 2");
            e->opt.lane_join = static_cast<uint32_t>(value);
            return HGX_OK;
        case HGX_OPT_EVENT_SIGNATURE_KEYS:
            if (value & ~uint64_t(0xF))
                return fail(HGX_ERR_INVALID,
                            "event signature keys: only input state (1), output state (2), step (4) "
                            "and rule (8) are provided; edge-rank keys need an exact canonical labelling");
            e->opt.event_keys = static_cast<uint32_t>(value);
            return HGX_OK;
    }
    return fail(HGX_ERR_INVALID, "unknown option");
}

hgx_status hgx_evolve(hgx_engine* e, const uint32_t* roots, size_t roots_len, uint32_t steps,
                      hgx_result** out) {
    if (!e || !roots || !out) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        if (e->rules.empty()) throw std::invalid_argument("evolve: no rules added");
        hgx::EvolutionSpec s;
        s.rules = e->rules;
        s.roots = read_roots(roots, roots_len);
        s.steps = steps;
        s.quotient = e->quotient;
        s.max_states = e->max_states;
        auto res = e->engine.run({s}, e->opt);
        *out = wrap(std::move(res[0]));
        return HGX_OK;
    });
}

hgx_status hgx_evolve_batch(hgx_engine* e, const hgx_job* jobs, uint32_t n, hgx_result** out) {
    if (!e || (!jobs && n) || (!out && n)) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        std::vector<hgx::EvolutionSpec> specs;
        specs.reserve(n);
        for (uint32_t i = 0; i < n; ++i) specs.push_back(spec_of(jobs[i]));
        auto res = e->engine.run(specs, e->opt);
        for (uint32_t i = 0; i < n; ++i) out[i] = wrap(std::move(res[i]));
        return HGX_OK;
    });
}

hgx_status hgx_serve_reset(hgx_engine* e) {
    if (!e) return fail(HGX_ERR_INVALID, "null engine");
    return guarded([&] {
        e->engine.reset();
        return HGX_OK;
    });
}

hgx_status hgx_serve_admit(hgx_engine* e, const hgx_job* job, uint32_t* id) {
    if (!e || !job || !id) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        *id = e->engine.admit(spec_of(*job));
        return HGX_OK;
    });
}

hgx_status hgx_serve_admit_batch(hgx_engine* e, const hgx_job* jobs, uint32_t n, uint32_t* ids) {
    if (!e || (n && (!jobs || !ids))) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        std::vector<hgx::EvolutionSpec> specs;
        specs.reserve(n);
        for (uint32_t i = 0; i < n; ++i) specs.push_back(spec_of(jobs[i]));
        const std::vector<uint32_t> got = e->engine.admit(specs);
        for (uint32_t i = 0; i < n; ++i) ids[i] = got[i];
        return HGX_OK;
    });
}

hgx_status hgx_serve_step(hgx_engine* e, int* still_active) {
    if (!e) return fail(HGX_ERR_INVALID, "null engine");
    return guarded([&] {
        const bool more = e->engine.step(e->opt);
        if (still_active) *still_active = more ? 1 : 0;
        return HGX_OK;
    });
}

hgx_status hgx_serve_take_finished(hgx_engine* e, uint32_t* ids, uint32_t cap, uint32_t* n) {
    if (!e || !n || (!ids && cap)) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        auto f = e->engine.take_finished();
        if (f.size() > cap) throw std::invalid_argument("take_finished: id buffer too small");
        std::memcpy(ids, f.data(), f.size() * sizeof(uint32_t));
        *n = static_cast<uint32_t>(f.size());
        return HGX_OK;
    });
}

hgx_status hgx_serve_collect_batch(hgx_engine* e, const uint32_t* ids, uint32_t n, hgx_result** out) {
    if (!e || (n && (!ids || !out))) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        auto res = e->engine.collect(std::vector<uint32_t>(ids, ids + n), e->opt);
        for (uint32_t i = 0; i < n; ++i) out[i] = wrap(std::move(res[i]));
        return HGX_OK;
    });
}

hgx_status hgx_serve_collect(hgx_engine* e, uint32_t evo, hgx_result** out) {
    if (!e || !out) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        *out = wrap(e->engine.collect(evo, e->opt));
        return HGX_OK;
    });
}

hgx_status hgx_serve_device_bytes(hgx_engine* e, uint64_t* bytes) {
    if (!e || !bytes) return fail(HGX_ERR_INVALID, "null argument");
    *bytes = e->engine.device_bytes_in_use();
    return HGX_OK;
}

hgx_status hgx_estimate_device_bytes(const hgx_job* job, uint64_t* bytes) {
    if (!job || !bytes) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        *bytes = hgx::Engine::estimate_bytes(spec_of(*job));
        return HGX_OK;
    });
}

hgx_status hgx_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    if (!free_bytes || !total_bytes) return fail(HGX_ERR_INVALID, "null argument");
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
            throw std::runtime_error("no CUDA device");
        if (device < 0 || device >= n) throw std::invalid_argument("device index out of range");
        int prev = 0;
        cudaError_t err = cudaGetDevice(&prev);
        if (err != cudaSuccess) throw hgx::CudaError(err, "cudaGetDevice", __FILE__, __LINE__);
        err = cudaSetDevice(device);
        if (err != cudaSuccess) throw hgx::CudaError(err, "cudaSetDevice", __FILE__, __LINE__);
        size_t f = 0, t = 0;
        err = cudaMemGetInfo(&f, &t);
        cudaSetDevice(prev);
        if (err != cudaSuccess) throw hgx::CudaError(err, "cudaMemGetInfo", __FILE__, __LINE__);
        *free_bytes = f;
        *total_bytes = t;
        return HGX_OK;
    });
}

uint64_t hgx_result_count(const hgx_result* res, hgx_count what) {
    if (!res) return 0;
    const auto& r = res->r;
    if (r.counts_only) {
        switch (what) {
            case HGX_COUNT_STATES: return r.n_states;
            case HGX_COUNT_EVENTS: return r.n_events;
            case HGX_COUNT_CLASSES: return r.num_classes;
            case HGX_COUNT_CAUSAL: return r.n_causal;
            case HGX_COUNT_BRANCHIAL: return r.n_branchial;
            case HGX_COUNT_TRUNCATED: return r.truncated ? 1 : 0;
            case HGX_COUNT_CANONICAL_EVENTS: return r.n_canonical_events;
            default: return 0;
        }
    }
    switch (what) {
        case HGX_COUNT_STATES: return res->count[HGX_ARR_STATE_HASH];
        case HGX_COUNT_EVENTS: return res->count[HGX_ARR_EVENTS] / 4;
        case HGX_COUNT_CLASSES: return r.num_classes;
        case HGX_COUNT_CAUSAL: return res->count[HGX_ARR_CAUSAL] / 3;
        case HGX_COUNT_BRANCHIAL: return res->count[HGX_ARR_BRANCHIAL] / 2;
        case HGX_COUNT_TRUNCATED: return r.truncated ? 1 : 0;
        case HGX_COUNT_CONSUMED: return res->count[HGX_ARR_EVENT_CONS];
        case HGX_COUNT_STATE_EDGES: return res->count[HGX_ARR_STATE_ARITY];
        case HGX_COUNT_STATE_VERTS: return res->count[HGX_ARR_STATE_VERTS];
        case HGX_COUNT_RAW_STATES: return r.n_roots + res->count[HGX_ARR_EVENTS] / 4;
        case HGX_COUNT_CANONICAL_EVENTS: return r.n_canonical_events;
    }
    return 0;
}

hgx_status hgx_result_copy(const hgx_result* res, hgx_array what, void* dst, size_t bytes) {
    if (!res || (!dst && bytes)) return fail(HGX_ERR_INVALID, "null argument");
    if (static_cast<int>(what) < 0 || static_cast<int>(what) >= hgx::ResultArrays::kArrays)
        return fail(HGX_ERR_INVALID, "unknown array");
    const size_t elem = (what == HGX_ARR_STATE_HASH || what == HGX_ARR_EVENT_SIG) ? 8
                        : what == HGX_ARR_STATE_ARITY                          ? 1
                                                                              : 4;
    const size_t need = res->count[what] * elem;
    if (bytes < need) return fail(HGX_ERR_INVALID, "hgx_result_copy: destination too small");
    if (need) std::memcpy(dst, res->ptr[what], need);
    return HGX_OK;
}

hgx_status hgx_result_view(const hgx_result* res, hgx_array what, const void** ptr, uint64_t* count) {
    if (!res || !ptr || !count) return fail(HGX_ERR_INVALID, "null argument");
    if (static_cast<int>(what) < 0 || static_cast<int>(what) >= hgx::ResultArrays::kArrays)
        return fail(HGX_ERR_INVALID, "unknown array");
    *ptr = res->ptr[what];
    *count = res->count[what];
    return HGX_OK;
}

hgx_status hgx_result_views(const hgx_result* res, const void** ptrs, uint64_t* counts) {
    if (!res || !ptrs || !counts) return fail(HGX_ERR_INVALID, "null argument");
    for (int i = 0; i < hgx::ResultArrays::kArrays; ++i) {
        ptrs[i] = res->ptr[i];
        counts[i] = res->count[i];
    }
    return HGX_OK;
}

void hgx_result_free(hgx_result* r) { delete r; }

hgx_status hgx_engine_stage_times(hgx_engine* e, double* out, uint64_t* launches) {
    if (!e || !out) return fail(HGX_ERR_INVALID, "null argument");
    const auto& t = e->engine.times();
    out[0] = t.count;
    out[1] = t.scan;
    out[2] = t.expand;
    out[3] = t.select;
    out[4] = t.materialize;
    out[5] = t.branchial;
    out[6] = t.roots;
    out[7] = t.count + t.scan + t.expand + t.expand_warp + t.select + t.materialize + t.branchial + t.roots;
    if (launches) *launches = t.launches;
    return HGX_OK;
}

hgx_status hgx_engine_expand_stats(hgx_engine* e, uint64_t* out) {
    if (!e || !out) return fail(HGX_ERR_INVALID, "null argument");
    const auto& t = e->engine.times();
    out[0] = t.expand_bytes;
    out[1] = t.expand_hbm_bytes;
    out[2] = t.children;
    out[3] = t.wl_rounds;
    out[4] = t.expand_launches;
    out[5] = t.warp_bytes;
    out[6] = t.warp_hbm_bytes;
    out[7] = t.warp_children;
    out[8] = t.warp_rounds;
    out[9] = static_cast<uint64_t>(t.expand_warp * 1e6);   // warp kernel time, ns
    out[10] = t.walk_launches;
    return HGX_OK;
}

hgx_status hgx_engine_result_stats(hgx_engine* e, uint64_t* out) {
    if (!e || !out) return fail(HGX_ERR_INVALID, "null argument");
    const auto& t = e->engine.times();
    out[0] = t.result_streamed;
    out[1] = t.result_chunks;
    return HGX_OK;
}

hgx_status hgx_engine_stream(hgx_engine* e, void** stream) {
    if (!e || !stream) return fail(HGX_ERR_INVALID, "null argument");
    *stream = reinterpret_cast<void*>(e->engine.stream());
    return HGX_OK;
}

}  // extern "C"
