// CPU restatement of the multiway evolution step -- TEST INFRASTRUCTURE ONLY (see restate.hpp).
//
// Reference anchors (paths inside the reference project):
//   hash primitives        common/include/hgcommon/core.hpp:47-87
//   WL canonical hash      common/include/hgcommon/wl_core.hpp:67-202
//   WL input convention    hypergraph/include/hypergraph/wl_hash.hpp:109-243 (sorted-unique local
//                          vertices, nbr_cap = max_v sum(arity-1), edges in ascending id order)
//   empty state hash       common/include/hgcommon/core.hpp:169, hypergraph/src/hypergraph.cpp:744
//   binding                common/include/hgcommon/match_core.hpp:32-49
//   the join               common/include/hgcommon/join_core.hpp:144-208
//   rewrite                common/include/hgcommon/rewrite_core.hpp:43-87, hypergraph/src/rewriter.cpp:11-117
//   causal triples         hypergraph/src/rewriter.cpp:138-191, hypergraph/src/causal_graph.cpp:187-228
//   branchial pairs        hypergraph/src/causal_graph.cpp:324-350
//   expansion policy       hypergraph/src/parallel_evolution.cpp:1697-1802 (full multiway: every raw
//                          state once; quotient: each class once at its shortest depth)
#include "restate.hpp"

#include <algorithm>
#include <map>
#include <set>
#include <cstring>
#include <functional>
#include <numeric>
#include <unordered_map>
#include <unordered_set>

namespace hgx_oracle {
namespace {

constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ULL;
constexpr uint64_t kFnvPrime = 0x100000001b3ULL;
constexpr uint64_t kEmptyStateHash = 0x9E3779B97F4A7C15ULL;
constexpr uint32_t kMaxRefine = 100;

inline uint64_t fnv(uint64_t h, uint64_t x) { return (h ^ x) * kFnvPrime; }

inline uint64_t smix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

uint32_t count_distinct(std::vector<uint64_t> c) {
    std::sort(c.begin(), c.end());
    return static_cast<uint32_t>(std::unique(c.begin(), c.end()) - c.begin());
}

}  // namespace

uint64_t wl_hash(const std::vector<std::vector<uint32_t>>& edges) {
    if (edges.empty()) return kEmptyStateHash;

    // Local vertex numbering. Any numbering gives the same hash (every fold below is either over
    // a sorted multiset or a commutative sum); sorted-unique is the reference adapter's choice.
    std::vector<uint32_t> verts;
    for (const auto& e : edges) verts.insert(verts.end(), e.begin(), e.end());
    std::sort(verts.begin(), verts.end());
    verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
    const uint32_t nv = static_cast<uint32_t>(verts.size());
    const uint32_t ne = static_cast<uint32_t>(edges.size());
    if (nv == 0) return 0;

    std::vector<std::vector<uint32_t>> ev(ne);
    for (uint32_t e = 0; e < ne; ++e)
        for (uint32_t v : edges[e])
            ev[e].push_back(static_cast<uint32_t>(
                std::lower_bound(verts.begin(), verts.end(), v) - verts.begin()));

    // Occurrences per vertex, in (edge, position) order, and the neighbour-list capacity
    // max_v sum(arity - 1) (at least 1).
    struct Occ { uint32_t e; uint32_t p; };
    std::vector<std::vector<Occ>> occ(nv);
    std::vector<uint32_t> nn(nv, 0);
    for (uint32_t e = 0; e < ne; ++e) {
        const uint32_t a = static_cast<uint32_t>(ev[e].size());
        for (uint32_t p = 0; p < a; ++p) {
            occ[ev[e][p]].push_back({e, p});
            nn[ev[e][p]] += a ? a - 1 : 0;
        }
    }
    uint32_t cap = 1;
    for (uint32_t v = 0; v < nv; ++v) cap = std::max(cap, nn[v]);

    // Initial colour: degree, then the (arity, position) pairs of the first `cap` occurrences,
    // sorted by the packed key (arity << 8 | position).
    std::vector<uint64_t> cur(nv), nxt(nv);
    for (uint32_t v = 0; v < nv; ++v) {
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(occ[v].size()));
        std::vector<uint64_t> keys;
        for (size_t j = 0; j < occ[v].size() && keys.size() < cap; ++j)
            keys.push_back((static_cast<uint64_t>(ev[occ[v][j].e].size()) << 8) | occ[v][j].p);
        std::sort(keys.begin(), keys.end());
        for (uint64_t k : keys) { h = fnv(h, k >> 8); h = fnv(h, k & 0xFFu); }
        cur[v] = h;
    }

    // Refinement: fold the sorted multiset {fnv(colour(u), k)} over every other position k of
    // every edge containing v. Stop once the distinct-colour count stops changing -- the colours
    // of the round that did not change the count are the ones kept.
    uint32_t prev = count_distinct(cur);
    for (uint32_t it = 0; it < kMaxRefine; ++it) {
        for (uint32_t v = 0; v < nv; ++v) {
            std::vector<uint64_t> nb;
            for (const Occ& o : occ[v])
                for (uint32_t k = 0; k < ev[o.e].size(); ++k)
                    if (k != o.p && nb.size() < cap) nb.push_back(fnv(cur[ev[o.e][k]], k));
            std::sort(nb.begin(), nb.end());
            uint64_t h = cur[v];
            for (uint64_t x : nb) h = fnv(h, x);
            nxt[v] = h;
        }
        cur.swap(nxt);
        const uint32_t d = count_distinct(cur);
        if (d == prev) break;
        prev = d;
    }

    // Connected components (a partition, so the labelling of roots is immaterial).
    std::vector<uint32_t> comp(nv);
    std::iota(comp.begin(), comp.end(), 0u);
    auto find = [&](uint32_t x) {
        while (comp[x] != x) x = comp[x] = comp[comp[x]];
        return x;
    };
    for (uint32_t e = 0; e < ne; ++e)
        for (size_t p = 1; p < ev[e].size(); ++p) {
            const uint32_t a = find(ev[e][0]), b = find(ev[e][p]);
            if (a != b) comp[std::max(a, b)] = std::min(a, b);
        }
    std::vector<uint64_t> csum_col(nv, 0), csize(nv, 0);
    for (uint32_t v = 0; v < nv; ++v) {
        const uint32_t r = find(v);
        csum_col[r] += smix(cur[v]);
        csize[r] += 1;
    }

    uint64_t vsum = 0, esum = 0, csum = 0;
    for (uint32_t v = 0; v < nv; ++v) vsum += smix(cur[v]);
    for (uint32_t e = 0; e < ne; ++e) {
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(ev[e].size()));
        for (uint32_t u : ev[e]) h = fnv(h, cur[u]);
        esum += smix(h);
        if (!ev[e].empty()) csize[find(ev[e][0])] += (uint64_t(1) << 32);
    }
    for (uint32_t v = 0; v < nv; ++v) {
        if (find(v) != v) continue;
        csum += smix(fnv(fnv(kFnvOffset, csize[v]), csum_col[v]));
    }
    uint64_t h = kFnvOffset;
    h = fnv(h, nv);
    h = fnv(h, ne);
    h = fnv(h, vsum);
    h = fnv(h, esum);
    h = fnv(h, csum);
    return h;
}

Rule make_rule(const std::vector<std::vector<uint8_t>>& lhs,
               const std::vector<std::vector<uint8_t>>& rhs) {
    Rule r;
    r.lhs = lhs;
    r.rhs = rhs;
    for (const auto& e : lhs) for (uint8_t v : e) r.lhs_mask |= 1u << v;
    for (const auto& e : rhs) for (uint8_t v : e) r.rhs_mask |= 1u << v;
    r.new_mask = r.rhs_mask & ~r.lhs_mask;
    // Binding schedule: position 0 first, then repeatedly the lowest-index position that shares
    // a variable with those already scheduled (the lowest unscheduled one if none does). Any
    // schedule finds the same match set; this one fixes the enumeration order, which is the
    // lexicographic order of the matched edges' positions taken in schedule order.
    const size_t k = lhs.size();
    std::vector<bool> used(k, false);
    uint32_t bound = 0;
    for (size_t step = 0; step < k; ++step) {
        size_t pick = k;
        for (size_t i = 0; i < k && pick == k; ++i) {
            if (used[i]) continue;
            uint32_t m = 0;
            for (uint8_t v : lhs[i]) m |= 1u << v;
            if (step == 0 || (m & bound)) pick = i;
        }
        if (pick == k)
            for (size_t i = 0; i < k; ++i) if (!used[i]) { pick = i; break; }
        used[pick] = true;
        for (uint8_t v : lhs[pick]) bound |= 1u << v;
        r.schedule.push_back(static_cast<uint8_t>(pick));
    }
    return r;
}

namespace {

struct Store {
    std::vector<std::vector<uint32_t>> edge_verts;
    std::vector<uint32_t> edge_creator;
    std::vector<std::vector<uint32_t>> state_edges;   // ascending edge ids
};

// All edge-injective, vertex-non-injective assignments of the LHS to the state's edges,
// enumerated depth-first in schedule order with candidates in ascending edge order.
void enumerate(const Store& st, const std::vector<uint32_t>& sedges, const Rule& r,
               std::vector<std::vector<uint32_t>>& out) {
    const size_t k = r.lhs.size();
    std::vector<uint32_t> binding(32, kNone);
    std::vector<uint32_t> matched(k, kNone);
    uint32_t mask = 0;
    std::vector<uint32_t> taken;
    std::function<void(size_t)> dfs = [&](size_t d) {
        if (d == k) { out.push_back(matched); return; }
        const uint8_t p = r.schedule[d];
        const auto& pat = r.lhs[p];
        for (uint32_t eid : sedges) {
            if (std::find(taken.begin(), taken.end(), eid) != taken.end()) continue;
            const auto& ev = st.edge_verts[eid];
            if (ev.size() != pat.size()) continue;
            const uint32_t saved = mask;
            bool ok = true;
            for (size_t i = 0; i < pat.size() && ok; ++i) {
                const uint32_t bit = 1u << pat[i];
                if (mask & bit) ok = binding[pat[i]] == ev[i];
                else { binding[pat[i]] = ev[i]; mask |= bit; }
            }
            if (ok) {
                matched[p] = eid;
                taken.push_back(eid);
                dfs(d + 1);
                taken.pop_back();
                matched[p] = kNone;
            }
            mask = saved;
        }
    };
    dfs(0);
}

// Re-derive the variable binding of a completed match.
void bind_all(const Store& st, const Rule& r, const std::vector<uint32_t>& m,
              std::vector<uint32_t>& binding) {
    binding.assign(32, kNone);
    for (size_t p = 0; p < r.lhs.size(); ++p)
        for (size_t i = 0; i < r.lhs[p].size(); ++i)
            binding[r.lhs[p][i]] = st.edge_verts[m[p]][i];
}

uint64_t hash_state(const Store& st, const std::vector<uint32_t>& sedges) {
    std::vector<std::vector<uint32_t>> e;
    e.reserve(sedges.size());
    for (uint32_t id : sedges) e.push_back(st.edge_verts[id]);
    return wl_hash(e);
}

}  // namespace

Result evolve(const std::vector<Rule>& rules,
              const std::vector<std::vector<std::vector<uint32_t>>>& roots, uint32_t steps,
              bool quotient, uint64_t max_states) {
    Result res;
    Store st;
    uint32_t next_vertex = 0;
    for (const auto& root : roots)
        for (const auto& e : root)
            for (uint32_t v : e) next_vertex = std::max(next_vertex, v + 1);

    std::unordered_map<uint64_t, uint32_t> cls;   // WL hash -> representative state
    std::vector<uint32_t> frontier;

    auto new_state = [&](std::vector<uint32_t>&& edges, uint64_t h, uint32_t depth) {
        const uint32_t sid = static_cast<uint32_t>(st.state_edges.size());
        st.state_edges.push_back(std::move(edges));
        res.state_hash.push_back(h);
        res.state_depth.push_back(depth);
        return sid;
    };

    for (const auto& root : roots) {
        std::vector<uint32_t> ids;
        for (const auto& e : root) {
            ids.push_back(static_cast<uint32_t>(st.edge_verts.size()));
            st.edge_verts.push_back(e);
            st.edge_creator.push_back(kNone);
        }
        const uint64_t h = hash_state(st, ids);
        const uint32_t sid = new_state(std::move(ids), h, 0);
        cls.emplace(h, sid);
        frontier.push_back(sid);
    }

    bool stop = false;
    for (uint32_t level = 0; level < steps && !stop && !frontier.empty(); ++level) {
        std::vector<uint32_t> next;
        for (uint32_t f : frontier) {
            if (stop) break;
            const uint32_t first_event = static_cast<uint32_t>(res.events.size());
            for (uint32_t ri = 0; ri < rules.size() && !stop; ++ri) {
                const Rule& r = rules[ri];
                std::vector<std::vector<uint32_t>> matches;
                enumerate(st, st.state_edges[f], r, matches);
                for (const auto& m : matches) {
                    // Child = parent - consumed + produced. Produced ids exceed every existing
                    // id, so appending keeps the list ascending.
                    std::vector<uint32_t> binding, fresh(32, kNone);
                    bind_all(st, r, m, binding);
                    for (uint32_t mask = r.new_mask; mask; mask &= mask - 1)
                        fresh[__builtin_ctz(mask)] = next_vertex++;
                    std::vector<uint32_t> child;
                    for (uint32_t id : st.state_edges[f])
                        if (std::find(m.begin(), m.end(), id) == m.end()) child.push_back(id);
                    std::vector<std::vector<uint32_t>> produced_verts;
                    for (const auto& pe : r.rhs) {
                        std::vector<uint32_t> vs;
                        for (uint8_t var : pe) vs.push_back(binding[var] != kNone ? binding[var] : fresh[var]);
                        produced_verts.push_back(vs);
                    }
                    // Hash the child before committing anything, so the state cap can refuse
                    // the event cleanly.
                    std::vector<std::vector<uint32_t>> cv;
                    for (uint32_t id : child) cv.push_back(st.edge_verts[id]);
                    for (const auto& pv : produced_verts) cv.push_back(pv);
                    const uint64_t h = wl_hash(cv);
                    const bool is_new_class = cls.find(h) == cls.end();
                    const uint64_t states_now = quotient ? cls.size() : res.state_hash.size();
                    const bool adds_state = quotient ? is_new_class : true;
                    if (max_states && adds_state && states_now >= max_states) {
                        res.truncated = true;
                        stop = true;
                        break;
                    }
                    const uint32_t eid = static_cast<uint32_t>(res.events.size());
                    Event ev;
                    ev.in_state = f;
                    ev.rule = ri;
                    ev.step = level + 1;
                    ev.out_hash = h;
                    ev.consumed = m;
                    for (const auto& pv : produced_verts) {
                        const uint32_t id = static_cast<uint32_t>(st.edge_verts.size());
                        st.edge_verts.push_back(pv);
                        st.edge_creator.push_back(eid);
                        ev.produced.push_back(id);
                        child.push_back(id);
                    }
                    if (!quotient || is_new_class) {
                        const uint32_t sid = new_state(std::move(child), h, level + 1);
                        if (is_new_class) cls.emplace(h, sid);
                        ev.out_state = sid;
                        next.push_back(sid);
                    } else {
                        ev.out_state = cls[h];
                    }
                    // Causal: every consumed edge with a producer gives (producer, this, edge).
                    for (uint32_t c : m)
                        if (st.edge_creator[c] != kNone) {
                            res.causal.push_back(st.edge_creator[c]);
                            res.causal.push_back(eid);
                            res.causal.push_back(c);
                        }
                    res.events.push_back(std::move(ev));
                }
            }
            // Branchial: events of this input state that consumed a common edge, each unordered
            // pair once.
            const uint32_t last_event = static_cast<uint32_t>(res.events.size());
            for (uint32_t a = first_event; a < last_event; ++a)
                for (uint32_t b = a + 1; b < last_event; ++b) {
                    bool share = false;
                    for (uint32_t x : res.events[a].consumed)
                        for (uint32_t y : res.events[b].consumed) share |= (x == y);
                    if (share) { res.branchial.push_back(a); res.branchial.push_back(b); }
                }
        }
        frontier.swap(next);
    }
    res.num_classes = cls.size();
    return res;
}

// Reachability restated directly: a pair (p, c) is implied when some other successor w of p
// reaches c. For each producer p the set of nodes reachable from p's successors is gathered by a
// depth-first walk over the unique-pair adjacency; a pair survives if c is not in that set.
std::vector<uint32_t> reduce_causal(const std::vector<uint32_t>& triples) {
    std::map<uint32_t, std::set<uint32_t>> succ;
    for (size_t i = 0; i + 2 < triples.size(); i += 3) succ[triples[i]].insert(triples[i + 1]);
    std::set<std::pair<uint32_t, uint32_t>> implied;
    for (const auto& [p, targets] : succ) {
        std::set<uint32_t> reach;          // reachable from p by a path of length >= 2
        std::vector<uint32_t> todo;
        for (uint32_t w : targets) {
            auto it = succ.find(w);
            if (it == succ.end()) continue;
            for (uint32_t x : it->second)
                if (reach.insert(x).second) todo.push_back(x);
        }
        while (!todo.empty()) {
            const uint32_t x = todo.back();
            todo.pop_back();
            auto it = succ.find(x);
            if (it == succ.end()) continue;
            for (uint32_t y : it->second)
                if (reach.insert(y).second) todo.push_back(y);
        }
        for (uint32_t c : targets)
            if (reach.count(c)) implied.insert({p, c});
    }
    std::vector<uint32_t> out;
    for (size_t i = 0; i + 2 < triples.size(); i += 3)
        if (!implied.count({triples[i], triples[i + 1]}))
            out.insert(out.end(), {triples[i], triples[i + 1], triples[i + 2]});
    return out;
}

}  // namespace hgx_oracle

// ---------------------------------------------------------------------------------------------
// Flat C interface for ctypes (tests, smoke, bench cpu_baseline).
//
// Blob encodings (uint32 arrays):
//   rules  [n_rules, per rule: n_lhs, (arity, vars...)*n_lhs, n_rhs, (arity, vars...)*n_rhs]
//   roots  [n_roots, per root: n_edges, (arity, vertices...)*n_edges]
// ---------------------------------------------------------------------------------------------
namespace {

struct Handle {
    hgx_oracle::Result r;
    std::vector<uint32_t> events_flat;   // in, out, rule, step
    std::vector<uint64_t> event_out_hash;
};

bool parse_rules(const uint32_t* b, size_t n, std::vector<hgx_oracle::Rule>& out) {
    size_t i = 0;
    auto get = [&](uint32_t& x) { if (i >= n) return false; x = b[i++]; return true; };
    uint32_t nr;
    if (!get(nr)) return false;
    for (uint32_t r = 0; r < nr; ++r) {
        std::vector<std::vector<uint8_t>> side[2];
        for (int s = 0; s < 2; ++s) {
            uint32_t ne;
            if (!get(ne)) return false;
            for (uint32_t e = 0; e < ne; ++e) {
                uint32_t a;
                if (!get(a)) return false;
                std::vector<uint8_t> vs(a);
                for (uint32_t k = 0; k < a; ++k) { uint32_t v; if (!get(v) || v >= 32) return false; vs[k] = static_cast<uint8_t>(v); }
                side[s].push_back(vs);
            }
        }
        out.push_back(hgx_oracle::make_rule(side[0], side[1]));
    }
    return true;
}

bool parse_roots(const uint32_t* b, size_t n, std::vector<std::vector<std::vector<uint32_t>>>& out) {
    size_t i = 0;
    auto get = [&](uint32_t& x) { if (i >= n) return false; x = b[i++]; return true; };
    uint32_t nroots;
    if (!get(nroots)) return false;
    for (uint32_t r = 0; r < nroots; ++r) {
        uint32_t ne;
        if (!get(ne)) return false;
        std::vector<std::vector<uint32_t>> st;
        for (uint32_t e = 0; e < ne; ++e) {
            uint32_t a;
            if (!get(a)) return false;
            std::vector<uint32_t> vs(a);
            for (uint32_t k = 0; k < a; ++k) if (!get(vs[k])) return false;
            st.push_back(vs);
        }
        out.push_back(st);
    }
    return true;
}

}  // namespace

extern "C" {

// WL hash of one hypergraph blob [n_edges, (arity, vertices...)*n_edges].
uint64_t oracle_wl_hash(const uint32_t* blob, size_t len) {
    std::vector<std::vector<std::vector<uint32_t>>> one;
    std::vector<uint32_t> tmp(len + 1);
    tmp[0] = 1;
    std::memcpy(tmp.data() + 1, blob, len * sizeof(uint32_t));
    if (!parse_roots(tmp.data(), tmp.size(), one) || one.empty()) return 0;
    return hgx_oracle::wl_hash(one[0]);
}

void* oracle_evolve(const uint32_t* rules, size_t rules_len, const uint32_t* roots,
                    size_t roots_len, uint32_t steps, int quotient, uint64_t max_states) {
    std::vector<hgx_oracle::Rule> rs;
    std::vector<std::vector<std::vector<uint32_t>>> rt;
    if (!parse_rules(rules, rules_len, rs) || !parse_roots(roots, roots_len, rt)) return nullptr;
    auto* h = new Handle;
    h->r = hgx_oracle::evolve(rs, rt, steps, quotient != 0, max_states);
    for (const auto& e : h->r.events) {
        h->events_flat.insert(h->events_flat.end(), {e.in_state, e.out_state, e.rule, e.step});
        h->event_out_hash.push_back(e.out_hash);
    }
    return h;
}

// Replace the handle's causal triples by their transitive reduction.
void oracle_reduce_causal(void* hp) {
    auto* h = static_cast<Handle*>(hp);
    h->r.causal = hgx_oracle::reduce_causal(h->r.causal);
}

// what: 0 states, 1 events, 2 causal triples, 3 branchial pairs, 4 classes, 5 truncated
uint64_t oracle_count(void* hp, int what) {
    auto* h = static_cast<Handle*>(hp);
    switch (what) {
        case 0: return h->r.state_hash.size();
        case 1: return h->r.events.size();
        case 2: return h->r.causal.size() / 3;
        case 3: return h->r.branchial.size() / 2;
        case 4: return h->r.num_classes;
        case 5: return h->r.truncated ? 1 : 0;
    }
    return 0;
}

// what: 0 state hashes (u64), 1 state depths (u32), 2 events (u32 x4), 3 causal (u32 x3),
//       4 branchial (u32 x2)
void oracle_copy(void* hp, int what, void* out) {
    auto* h = static_cast<Handle*>(hp);
    switch (what) {
        case 0: std::memcpy(out, h->r.state_hash.data(), h->r.state_hash.size() * 8); break;
        case 1: std::memcpy(out, h->r.state_depth.data(), h->r.state_depth.size() * 4); break;
        case 2: std::memcpy(out, h->events_flat.data(), h->events_flat.size() * 4); break;
        case 3: std::memcpy(out, h->r.causal.data(), h->r.causal.size() * 4); break;
        case 4: std::memcpy(out, h->r.branchial.data(), h->r.branchial.size() * 4); break;
    }
}

void oracle_free(void* hp) { delete static_cast<Handle*>(hp); }

}  // extern "C"
