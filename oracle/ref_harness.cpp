// Reference-engine harness (test infrastructure; never part of the product path).
//
// Links the reference CPU engine's own sources, unmodified and compiled where they lie, and
// runs one evolution described by a small text spec. It prints one JSON object with the
// normalised result that the parity tests compare against:
//
//   * WL mode = StateCanonicalizationMode::None with the reported per-state canonical hash,
//     which is the WL hash (hypergraph/src/hypergraph.cpp:180-197, :618-626, :740-755).
//     Event keys, causal keys and branchial keys follow the reference's own cross-engine
//     normalisation (gpu/tests/test_gpu_vs_cpu_differential.cpp:119-157, applied at :276-321).
//   * quotient mode = StateCanonicalizationMode::Full with explore_from_canonical_states_only
//     (IR-keyed; the reference has no WL-keyed quotient, parallel_evolution.cpp:1471-1476).
//     Only counts are reported there: they pin the WL-quotient restatement wherever the WL
//     classes coincide with the IR classes.
//
// Spec (whitespace separated, read from the file named by argv[1]):
//   steps <n>
//   mode full|quotient
//   threads <n>            0 = serial execution mode (deterministic ids)
//   rule <nl> (<a> v..)*nl <nr> (<a> v..)*nr      (repeatable)
//   root <ne> (<a> v..)*ne                        (repeatable: several roots)
//   arrays 0|1             1 = also print the full sorted key arrays
//   tr 0|1                 transitive reduction of the causal graph (default 0)
//   evkeys <bits>          event signature keys (hgcommon EventSignatureKeys; default 0 = none):
//                          then "events" is the canonical event count and "signature_digest" the
//                          digest of the sorted distinct signatures of the canonical events
#include <hypergraph/hypergraph.hpp>
#include <hypergraph/parallel_evolution.hpp>
#include <hypergraph/pattern.hpp>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

using namespace hypergraph;

namespace {

constexpr uint64_t kOffset = 14695981039346656037ULL;
constexpr uint64_t kPrime = 1099511628211ULL;

uint64_t fold(uint64_t h, uint64_t x) { return (h ^ x) * kPrime; }

uint64_t event_key(uint64_t in_h, uint64_t out_h, uint64_t rule, uint64_t step) {
    return fold(fold(fold(fold(kOffset, in_h), out_h), rule), step);
}
uint64_t pair_key_unordered(uint64_t a, uint64_t b) {
    return fold(fold(kOffset, std::min(a, b)), std::max(a, b));
}
uint64_t pair_key_directed(uint64_t a, uint64_t b) { return fold(fold(kOffset, a), b); }

uint64_t digest(const std::vector<uint64_t>& sorted) {
    uint64_t h = kOffset;
    for (uint64_t x : sorted) h = fold(h, x);
    return fold(h, sorted.size());
}

struct Spec {
    int steps = 0;
    bool quotient = false;
    int threads = 0;
    bool arrays = false;
    bool tr = false;
    int evkeys = 0;
    std::vector<std::pair<std::vector<std::vector<uint8_t>>, std::vector<std::vector<uint8_t>>>> rules;
    std::vector<std::vector<std::vector<VertexId>>> roots;
};

bool read_spec(const char* path, Spec& s) {
    std::ifstream in(path);
    if (!in) return false;
    std::string tok;
    auto read_edges_u8 = [&](std::vector<std::vector<uint8_t>>& out) {
        int n; in >> n;
        for (int i = 0; i < n; ++i) {
            int a; in >> a;
            std::vector<uint8_t> e(a);
            for (int k = 0; k < a; ++k) { int v; in >> v; e[k] = static_cast<uint8_t>(v); }
            out.push_back(e);
        }
    };
    while (in >> tok) {
        if (tok == "steps") in >> s.steps;
        else if (tok == "mode") { std::string m; in >> m; s.quotient = (m == "quotient"); }
        else if (tok == "threads") in >> s.threads;
        else if (tok == "arrays") { int a; in >> a; s.arrays = a != 0; }
        else if (tok == "tr") { int a; in >> a; s.tr = a != 0; }
        else if (tok == "evkeys") in >> s.evkeys;
        else if (tok == "rule") {
            std::vector<std::vector<uint8_t>> l, r;
            read_edges_u8(l);
            read_edges_u8(r);
            s.rules.emplace_back(l, r);
        } else if (tok == "root") {
            int n; in >> n;
            std::vector<std::vector<VertexId>> st;
            for (int i = 0; i < n; ++i) {
                int a; in >> a;
                std::vector<VertexId> e(a);
                for (int k = 0; k < a; ++k) { long long v; in >> v; e[k] = static_cast<VertexId>(v); }
                st.push_back(e);
            }
            s.roots.push_back(st);
        } else {
            std::fprintf(stderr, "unknown token %s\n", tok.c_str());
            return false;
        }
    }
    return true;
}

void print_array(const char* name, const std::vector<uint64_t>& v) {
    std::printf(",\"%s\":[", name);
    for (size_t i = 0; i < v.size(); ++i) std::printf(i ? ",%llu" : "%llu", (unsigned long long)v[i]);
    std::printf("]");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: hgref <spec>\n"); return 2; }
    Spec spec;
    if (!read_spec(argv[1], spec) || spec.rules.empty() || spec.roots.empty()) {
        std::fprintf(stderr, "bad spec\n");
        return 2;
    }

    Hypergraph hg;
    hg.set_state_canonicalization_mode(spec.quotient ? StateCanonicalizationMode::Full
                                                     : StateCanonicalizationMode::None);
    const auto mode = spec.threads == 0 ? ParallelEvolutionEngine::ExecutionMode::Serial
                                        : ParallelEvolutionEngine::ExecutionMode::Parallel;
    ParallelEvolutionEngine engine(&hg, static_cast<size_t>(spec.threads), mode);
    hg.set_event_signature_keys(static_cast<hgcommon::EventSignatureKeys>(spec.evkeys));
    engine.set_transitive_reduction(spec.tr);
    engine.set_explore_from_canonical_states_only(spec.quotient);
    for (size_t i = 0; i < spec.rules.size(); ++i) {
        RuleBuilder b(static_cast<uint16_t>(i));
        for (const auto& e : spec.rules[i].first) b.lhs(e);
        for (const auto& e : spec.rules[i].second) b.rhs(e);
        engine.add_rule(b.build());
    }

    const auto t0 = std::chrono::steady_clock::now();
    if (spec.roots.size() == 1) engine.evolve(spec.roots[0], static_cast<size_t>(spec.steps));
    else engine.evolve(spec.roots, static_cast<size_t>(spec.steps));
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    const uint32_t n_states = hg.num_states();
    const uint32_t n_events = hg.num_events();
    std::printf("{\"raw_states\":%u,\"events\":%u,\"canonical_states\":%zu,\"ms\":%.3f,\"threads\":%d",
                n_states, n_events, hg.num_canonical_states(), ms, spec.threads);

    if (!spec.quotient) {
        std::vector<uint64_t> hash_of(n_states, 0);
        std::set<uint64_t> classes;
        for (uint32_t s = 0; s < n_states; ++s) {
            hash_of[s] = hg.get_or_compute_canonical_hash(s);
            classes.insert(hash_of[s]);
        }
        std::unordered_map<uint32_t, uint64_t> key_of;
        std::vector<uint64_t> ekeys;
        std::set<uint64_t> sigs;
        for (uint32_t e = 0; e < hg.num_published_events(); ++e) {
            const auto& ev = hg.get_event(e);
            if (ev.id == INVALID_ID) continue;
            if (spec.evkeys && hg.get_canonical_event(e) == e) sigs.insert(ev.signature);
            const uint32_t step = hg.get_state(ev.output_state).step;
            const uint64_t k = event_key(hash_of[ev.input_state], hash_of[ev.output_state],
                                         ev.rule_index, step);
            key_of[e] = k;
            ekeys.push_back(k);
        }
        std::vector<uint64_t> ckeys, bkeys;
        for (const auto& ce : hg.causal_graph().get_causal_edges()) {
            auto p = key_of.find(ce.producer), c = key_of.find(ce.consumer);
            if (p == key_of.end() || c == key_of.end()) continue;
            ckeys.push_back(pair_key_directed(p->second, c->second));
        }
        for (const auto& be : hg.causal_graph().get_branchial_edges()) {
            auto a = key_of.find(be.event1), b = key_of.find(be.event2);
            if (a == key_of.end() || b == key_of.end()) continue;
            bkeys.push_back(pair_key_unordered(a->second, b->second));
        }
        std::sort(ekeys.begin(), ekeys.end());
        std::sort(ckeys.begin(), ckeys.end());
        std::sort(bkeys.begin(), bkeys.end());
        std::vector<uint64_t> hs(classes.begin(), classes.end());
        std::printf(",\"wl_classes\":%zu,\"causal\":%zu,\"branchial\":%zu", hs.size(), ckeys.size(),
                    bkeys.size());
        std::printf(",\"event_digest\":%llu,\"causal_digest\":%llu,\"branchial_digest\":%llu",
                    (unsigned long long)digest(ekeys), (unsigned long long)digest(ckeys),
                    (unsigned long long)digest(bkeys));
        if (spec.evkeys) {
            std::vector<uint64_t> sv(sigs.begin(), sigs.end());
            std::printf(",\"raw_events\":%u,\"signatures\":%zu,\"signature_digest\":%llu",
                        hg.num_raw_events(), sv.size(), (unsigned long long)digest(sv));
        }
        print_array("state_hashes", hs);
        if (spec.arrays) {
            print_array("event_keys", ekeys);
            print_array("causal_keys", ckeys);
            print_array("branchial_keys", bkeys);
        }
    }
    std::printf("}\n");
    return 0;
}
