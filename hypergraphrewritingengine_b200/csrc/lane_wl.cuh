// Lane-per-child WL canonical hash (one thread hashes one child against its parent).
//
// Host and device: the same function runs in the expand kernel and in the native unit test
// (tests/native/lane_wl_test.cpp), which checks it against the oracle's WL hash on random
// parents and matches.
//
// A child is given relative to its parent: the parent's edges (arity pear[e], vertex offset
// pevo[e] into vloc), the parent's per-vertex occurrence lists in edge order (poff/pocc, entries
// e << 4 | position), per-vertex degree pdeg and neighbour count pnn (sum of arity - 1), the
// parent's per-vertex neighbour lists (pnoff/pnbr, entries lane_nbr_entry(e, u, k): vertex u at
// position k of edge e, one per other position of every occurrence), and a slot holding the
// parent positions the match removes (pattern order) followed by the local vertex ids of the
// produced edges (RHS order). Local ids: parent vertices [0, nvp), the n-th
// fresh variable nvp + n. The child's edge order is the parent's minus the removed edges,
// then the produced ones -- the order the reference hashes a state's edges in.
//
// The arithmetic restates common/include/hgcommon/wl_core.hpp:67-202 of the reference: initial
// colour FNV(degree, sorted (arity, position) of the first `cap` occurrences), refinement by the
// sorted multiset of fnv(colour(u), k) until the distinct-colour count stops changing (at most
// 100 rounds), then the connected-component fold and FNV(n_v, n_e, vsum, esum, csum).
#pragma once
#include "common.cuh"

namespace hgx {

struct WlInfo {
    uint32_t rounds, nv, nocc, nbr;   // refinement rounds run, vertices, occurrences, sum a(a-1)
};

// One neighbour entry of a parent vertex: the edge it comes from (< 64, tested against the removed
// positions), the neighbour's local id (< 64) and its position in that edge (< 16).
HGX_HD uint16_t lane_nbr_entry(uint32_t e, uint32_t u, uint32_t k) {
    return static_cast<uint16_t>((e << 10) | (u << 4) | k);
}

HGX_HD uint32_t lane_ctz64(uint64_t m) {
#ifdef __CUDA_ARCH__
    return static_cast<uint32_t>(__ffsll(static_cast<long long>(m)) - 1);
#else
    return static_cast<uint32_t>(__builtin_ctzll(m));
#endif
}

// Host form of the parent neighbour lists (the expand kernel builds them warp-parallel).
inline void lane_build_nbr(const uint8_t* pear, const uint16_t* pevo, const uint16_t* vloc,
                           uint32_t pne, uint32_t nvp, uint16_t* pnoff, uint16_t* pnbr) {
    uint32_t w = 0;
    for (uint32_t v = 0; v < nvp; ++v) {
        pnoff[v] = static_cast<uint16_t>(w);
        for (uint32_t e = 0; e < pne; ++e)
            for (uint32_t q = 0; q < pear[e]; ++q) {
                if (vloc[pevo[e] + q] != v) continue;
                for (uint32_t k = 0; k < pear[e]; ++k)
                    if (k != q) pnbr[w++] = lane_nbr_entry(e, vloc[pevo[e] + k], k);
            }
    }
    pnoff[nvp] = static_cast<uint16_t>(w);
}

HGX_HD void lane_isort64(uint64_t* a, uint32_t n) {
        #pragma unroll 1
    for (uint32_t i = 1; i < n; ++i) {
        const uint64_t k = a[i];
        uint32_t j = i;
        while (j > 0 && a[j - 1] > k) { a[j] = a[j - 1]; --j; }
        a[j] = k;
    }
}

template <int VM>
HGX_HD uint32_t lane_distinct(const uint64_t* cur, uint32_t alive, uint32_t V) {
    uint32_t d = 0;
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) {
        if (!((alive >> v) & 1u)) continue;
        bool first = true;
                #pragma unroll 1
        for (uint32_t u = 0; u < v && first; ++u)
            if (((alive >> u) & 1u) && cur[u] == cur[v]) first = false;
        d += first ? 1u : 0u;
    }
    return d;
}

// Component term of a connected child.
HGX_HD uint64_t lane_one_component(uint32_t ne, uint32_t nv, uint64_t vs) {
    return smix(fnv(fnv(kFnvOffset, (static_cast<uint64_t>(ne) << 32) | nv), vs));
}

// Component term of a child whose connectivity is not known from its parent: union-find over its
// edges, then per component smix(fnv(fnv(offset, edges << 32 | vertices), sum of vertex terms)).
// Kept out of line: the expand kernel's hot path (connected children) stays small.
template <int VM>
HGX_NOINLINE uint64_t lane_component_term(const uint8_t* pear, const uint16_t* pevo,
                                          const uint16_t* vloc, uint32_t pne, const DevRule& R,
                                          const uint8_t* prodv, uint64_t rmask,
                                          uint32_t alive, const uint64_t* vterm, uint32_t V,
                                          uint32_t ne, uint32_t nv, uint64_t vs) {
    uint8_t comp[VM];
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) comp[v] = static_cast<uint8_t>(v);
    auto find = [&](uint32_t x) -> uint32_t {
        while (comp[x] != x) { comp[x] = comp[comp[x]]; x = comp[x]; }
        return x;
    };
        #pragma unroll 1
    for (uint32_t e = 0; e < pne; ++e) {
        if ((rmask >> e) & 1ull) continue;
        const uint32_t a = pear[e], vo = pevo[e];
        const uint32_t r = find(vloc[vo]);
                #pragma unroll 1
        for (uint32_t q = 1; q < a; ++q) {
            const uint32_t x = find(vloc[vo + q]);
            if (x != r) comp[x] = static_cast<uint8_t>(r);
        }
    }
        #pragma unroll 1
    for (uint32_t k = 0; k < R.n_rhs; ++k) {
        const uint32_t a = R.rhs_ar[k], o = R.rhs_off[k];
        const uint32_t r = find(prodv[o]);
                #pragma unroll 1
        for (uint32_t q = 1; q < a; ++q) {
            const uint32_t x = find(prodv[o + q]);
            if (x != r) comp[x] = static_cast<uint8_t>(r);
        }
    }
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) comp[v] = static_cast<uint8_t>(find(v));
    uint32_t roots = 0;
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) roots += (((alive >> v) & 1u) && comp[v] == v) ? 1u : 0u;
    if (roots == 1) return lane_one_component(ne, nv, vs);
    uint64_t cs = 0;
        #pragma unroll 1
    for (uint32_t r = 0; r < V; ++r) {
        if (!((alive >> r) & 1u) || comp[r] != r) continue;
        uint64_t col = 0, vc = 0, ec = 0;
                #pragma unroll 1
        for (uint32_t v = 0; v < V; ++v)
            if (((alive >> v) & 1u) && comp[v] == r) { col += vterm[v]; ++vc; }
                #pragma unroll 1
        for (uint32_t e = 0; e < pne; ++e)
            if (!((rmask >> e) & 1ull) && comp[vloc[pevo[e]]] == r) ++ec;
                #pragma unroll 1
        for (uint32_t k = 0; k < R.n_rhs; ++k)
            if (comp[prodv[R.rhs_off[k]]] == r) ++ec;
        cs += smix(fnv(fnv(kFnvOffset, (ec << 32) | vc), col));
    }
    return cs;
}

// Occurrence count of a packed per-position count word (one byte per position).
HGX_HD uint32_t lane_bytesum(uint32_t c) { return (c * 0x01010101u) >> 24; }

// pinfo: bit 0 = the parent is connected; bits 8.. = A when every parent edge has arity A (2..4),
// else 0. With A set and every RHS edge of arity A too (R.rhs_uni == A), a vertex's initial
// colour follows from its occurrence counts per position (pcnt: byte q = occurrences at position
// q), since the sorted (arity, position) multiset is then the positions in ascending order with
// their multiplicities, and no truncation applies (every vertex has at least as many neighbour
// entries as occurrences when A >= 2).
template <int VM, int NM>
HGX_HD uint64_t lane_wl_core(const uint8_t* pear, const uint16_t* pevo, const uint16_t* vloc,
                             const uint16_t* poff, const uint16_t* pocc, const uint16_t* pdeg,
                             const uint16_t* pnn, const uint16_t* pnoff, const uint16_t* pnbr,
                             const uint32_t* pcnt, uint32_t pinfo, uint32_t pne, uint32_t nvp,
                             const DevRule& R, const uint8_t* slot, WlInfo& info) {
    const uint8_t* rpos = slot;
    const uint8_t* prodv = slot + R.n_lhs;
    const uint32_t V = nvp + R.n_fresh;
    const uint32_t ne = pne - R.n_lhs + R.n_rhs;
    const bool pconn = (pinfo & 1u) != 0;
    const uint32_t A = (pinfo >> 8) == R.rhs_uni ? (pinfo >> 8) : 0u;   // uniform arity, or 0
    info.rounds = info.nv = info.nocc = info.nbr = 0;
    if (ne == 0) return kEmptyStateHash;

    uint64_t rmask = 0;
        #pragma unroll 1
    for (uint32_t k = 0; k < R.n_lhs; ++k) rmask |= 1ull << rpos[k];
    // uniform arity: occurrences by position (byte q); otherwise degree | neighbour count << 16
    uint32_t dn[VM];
    if (A) {
                #pragma unroll 1
        for (uint32_t v = 0; v < V; ++v) dn[v] = v < nvp ? pcnt[v] : 0u;
                #pragma unroll 1
        for (uint32_t k = 0; k < R.n_lhs; ++k) {
            const uint32_t vo = pevo[rpos[k]];
                        #pragma unroll 1
            for (uint32_t q = 0; q < A; ++q) dn[vloc[vo + q]] -= 1u << (8 * q);
        }
                #pragma unroll 1
        for (uint32_t p = 0; p < R.rhs_total; ++p) dn[prodv[p]] += 1u << (8 * (p % A));
    } else {
                #pragma unroll 1
        for (uint32_t v = 0; v < V; ++v) dn[v] = v < nvp ? (pdeg[v] | (uint32_t(pnn[v]) << 16)) : 0u;
                #pragma unroll 1
        for (uint32_t k = 0; k < R.n_lhs; ++k) {
            const uint32_t e = rpos[k], a = pear[e], vo = pevo[e];
                        #pragma unroll 1
            for (uint32_t q = 0; q < a; ++q) {
                const uint32_t v = vloc[vo + q];
                dn[v] -= 1u + ((a - 1u) << 16);
            }
        }
                #pragma unroll 1
        for (uint32_t k = 0; k < R.n_rhs; ++k) {
            const uint32_t a = R.rhs_ar[k], o = R.rhs_off[k];
                        #pragma unroll 1
            for (uint32_t q = 0; q < a; ++q) {
                const uint32_t v = prodv[o + q];
                dn[v] += 1u + ((a - 1u) << 16);
            }
        }
    }
    uint32_t nv = 0, cap = 1, nocc = 0, nbr = 0, alive = 0;   // alive: vertices of degree > 0
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) {
        const uint32_t d = A ? lane_bytesum(dn[v]) : dn[v] & 0xFFFFu;
        const uint32_t m = A ? d * (A - 1u) : dn[v] >> 16;
        nv += d ? 1u : 0u;
        alive |= (d ? 1u : 0u) << v;
        cap = m > cap ? m : cap;
        nocc += d;
        nbr += m;
    }
    info.nv = nv;
    info.nocc = nocc;
    info.nbr = nbr;
    if (nv == 0) return 0;
    // produced occurrences by vertex: bit p of pm[v] <=> RHS position p holds v (ascending p is
    // RHS edge order, then position order)
    uint64_t pm[VM];
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) pm[v] = 0;
        #pragma unroll 1
    for (uint32_t p = 0; p < R.rhs_total; ++p) pm[prodv[p]] |= 1ull << p;

    uint64_t cura[VM], curb[VM], buf[NM];
    uint64_t* cur = cura;   // this round's colours
    uint64_t* nxt = curb;   // the next round's (the two swap every round)
    // initial colours
    if (A) {
                #pragma unroll 1
        for (uint32_t v = 0; v < V; ++v) {
            const uint32_t c = dn[v];
            uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(lane_bytesum(c)));
                        #pragma unroll 1
            for (uint32_t q = 0; q < A; ++q) {
                                #pragma unroll 1
                for (uint32_t j = (c >> (8 * q)) & 0xFFu; j; --j) h = fnv(fnv(h, A), q);
            }
            cur[v] = ((alive >> v) & 1u) ? h : 0;
        }
    }
        #pragma unroll 1
    for (uint32_t v = 0; v < V && !A; ++v) {
        cur[v] = 0;
        if (!((alive >> v) & 1u)) continue;
        uint32_t n = 0;
        const uint32_t j0 = v < nvp ? poff[v] : 0u, j1 = v < nvp ? poff[v + 1] : 0u;
                #pragma unroll 1
        for (uint32_t j = j0; j < j1 && n < cap; ++j) {
            const uint32_t x = pocc[j], e = x >> 4;
            if ((rmask >> e) & 1ull) continue;
            buf[n++] = (static_cast<uint64_t>(pear[e]) << 8) | (x & 15u);
        }
                #pragma unroll 1
        for (uint64_t m = pm[v]; m && n < cap; m &= m - 1) {
            const uint32_t p = lane_ctz64(m), k = R.rhs_pos_edge[p];
            buf[n++] = (static_cast<uint64_t>(R.rhs_ar[k]) << 8) | (p - R.rhs_off[k]);
        }
        lane_isort64(buf, n);
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(dn[v] & 0xFFFFu));
                #pragma unroll 1
        for (uint32_t j = 0; j < n; ++j) {
            h = fnv(h, buf[j] >> 8);
            h = fnv(h, buf[j] & 0xFFu);
        }
        cur[v] = h;
    }
    uint32_t prev = lane_distinct<VM>(cur, alive, V);
        #pragma unroll 1
    for (uint32_t it = 0; it < kWlMaxRounds; ++it) {
                #pragma unroll 1
        for (uint32_t v = 0; v < V; ++v) {
            if (!((alive >> v) & 1u)) { nxt[v] = 0; continue; }
            // the neighbour multiset; nn[v] <= cap entries, so the reference's cap never cuts here
            uint32_t n = 0;
            const uint32_t j0 = v < nvp ? pnoff[v] : 0u, j1 = v < nvp ? pnoff[v + 1] : 0u;
                        #pragma unroll 1
            for (uint32_t j = j0; j < j1; ++j) {
                const uint32_t x = pnbr[j];
                if ((rmask >> (x >> 10)) & 1ull) continue;
                buf[n++] = fnv(cur[(x >> 4) & 63u], x & 15u);
            }
                        #pragma unroll 1
            for (uint64_t m = pm[v]; m; m &= m - 1) {
                const uint32_t p = lane_ctz64(m), kk = R.rhs_pos_edge[p];
                const uint32_t a = R.rhs_ar[kk], o = R.rhs_off[kk], q = p - o;
                                #pragma unroll 1
                for (uint32_t t = 0; t < a; ++t)
                    if (t != q) buf[n++] = fnv(cur[prodv[o + t]], t);
            }
            lane_isort64(buf, n);
            uint64_t h = cur[v];
                        #pragma unroll 1
            for (uint32_t j = 0; j < n; ++j) h = fnv(h, buf[j]);
            nxt[v] = h;
        }
        uint64_t* t = cur;
        cur = nxt;
        nxt = t;
        const uint32_t d = lane_distinct<VM>(cur, alive, V);
        ++info.rounds;
        if (d == prev) break;
        prev = d;
    }

    // the commutative folds, then the component term: a connected parent and a rule whose RHS
    // joins every LHS vertex give a connected child (one component, no partition needed)
    uint64_t vs = 0, es = 0;
        #pragma unroll 1
    for (uint32_t v = 0; v < V; ++v) {
        nxt[v] = ((alive >> v) & 1u) ? smix(cur[v]) : 0;
        vs += nxt[v];
    }
        #pragma unroll 1
    for (uint32_t e = 0; e < pne; ++e) {
        if ((rmask >> e) & 1ull) continue;
        const uint32_t a = pear[e], vo = pevo[e];
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(a));
                #pragma unroll 1
        for (uint32_t q = 0; q < a; ++q) h = fnv(h, cur[vloc[vo + q]]);
        es += smix(h);
    }
        #pragma unroll 1
    for (uint32_t k = 0; k < R.n_rhs; ++k) {
        const uint32_t a = R.rhs_ar[k], o = R.rhs_off[k];
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(a));
                #pragma unroll 1
        for (uint32_t q = 0; q < a; ++q) h = fnv(h, cur[prodv[o + q]]);
        es += smix(h);
    }
    const bool one = pconn && (R.flags & kRuleRhsJoinsLhs);
    const uint64_t cs = one ? lane_one_component(ne, nv, vs)
                            : lane_component_term<VM>(pear, pevo, vloc, pne, R, prodv, rmask, alive,
                                                      nxt, V, ne, nv, vs);
    uint64_t h = kFnvOffset;
    h = fnv(h, nv);
    h = fnv(h, ne);
    h = fnv(h, vs);
    h = fnv(h, es);
    h = fnv(h, cs);
    return h;
}


}  // namespace hgx
