// Native unit test of the expand kernel's lane-per-child WL (hypergraphrewritingengine_b200/
// csrc/lane_wl.cuh), compiled for the host: random parents and random matches, each child's
// hash checked against the oracle's WL hash of the explicitly built child. Exit 0 = all equal.
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include "../../hypergraphrewritingengine_b200/csrc/lane_wl.cuh"
#include "../../oracle/restate.hpp"

using namespace hgx;

int main(int argc, char** argv) {
    const int trials = argc > 1 ? atoi(argv[1]) : 20000;
    std::mt19937_64 rng(12345);
    auto U = [&](int lo, int hi) { return lo + int(rng() % uint64_t(hi - lo + 1)); };
    int fails = 0, shortcut = 0, uniform = 0;
    for (int t = 0; t < trials; ++t) {
        // parent: ne edges of arity in [amin, amax] over nverts labels
        const int amin = U(1, 3), amax = amin + U(0, 2);
        const int ne = U(2, 40), nverts = U(1, 12);
        std::vector<std::vector<uint32_t>> par(ne);
        for (auto& e : par) {
            e.resize(U(amin, amax));
            for (auto& v : e) v = 100 + U(0, nverts - 1);
        }
        // local ids by first occurrence, edge offsets, occurrence lists by vertex
        std::vector<uint8_t> pear(ne);
        std::vector<uint16_t> pevo(ne), vloc;
        std::vector<uint32_t> glob;
        for (int e = 0; e < ne; ++e) {
            pear[e] = uint8_t(par[e].size());
            pevo[e] = uint16_t(glob.size());
            for (uint32_t v : par[e]) glob.push_back(v);
        }
        std::vector<uint32_t> ids;
        for (uint32_t v : glob) {
            uint32_t k = 0;
            while (k < ids.size() && ids[k] != v) ++k;
            if (k == ids.size()) ids.push_back(v);
            vloc.push_back(uint16_t(k));
        }
        const uint32_t nvp = uint32_t(ids.size());
        std::vector<uint16_t> poff(nvp + 1, 0), pocc, pdeg(nvp, 0), pnn(nvp, 0);
        for (uint32_t v = 0; v < nvp; ++v) {
            poff[v] = uint16_t(pocc.size());
            for (int e = 0; e < ne; ++e)
                for (int q = 0; q < pear[e]; ++q)
                    if (vloc[pevo[e] + q] == v) {
                        pocc.push_back(uint16_t((e << 4) | q));
                        pdeg[v]++;
                        pnn[v] += pear[e] - 1;
                    }
        }
        poff[nvp] = uint16_t(pocc.size());
        std::vector<uint16_t> pnoff(nvp + 1, 0), pnbr(pocc.size() * 16);
        lane_build_nbr(pear.data(), pevo.data(), vloc.data(), uint32_t(ne), nvp, pnoff.data(), pnbr.data());
        // a "match": n_lhs distinct removed positions; produced edges over parent + fresh
        DevRule R;
        std::memset(&R, 0, sizeof(R));
        R.n_lhs = uint8_t(U(0, std::min(ne, 4)));
        R.n_rhs = uint8_t(U(0, 4));
        R.n_fresh = uint8_t(U(0, 2));
        std::vector<uint8_t> slot;
        std::vector<int> perm(ne);
        for (int i = 0; i < ne; ++i) perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        for (int k = 0; k < R.n_lhs; ++k) slot.push_back(uint8_t(perm[k]));
        uint32_t off = 0;
        std::vector<std::vector<uint32_t>> prod;
        for (int k = 0; k < R.n_rhs; ++k) {
            const int a = U(amin, amax);
            R.rhs_ar[k] = uint8_t(a);
            R.rhs_off[k] = uint8_t(off);
            for (int q = 0; q < a; ++q) R.rhs_pos_edge[off + q] = uint8_t(k);
            std::vector<uint32_t> pe;
            for (int q = 0; q < a; ++q) {
                const uint32_t lv = uint32_t(U(0, int(nvp + R.n_fresh) - 1));
                slot.push_back(uint8_t(lv));
                pe.push_back(lv < nvp ? ids[lv] : 5000 + lv);
            }
            prod.push_back(pe);
            off += a;
        }
        R.rhs_total = uint8_t(off);
        // explicit child in the reference's edge order
        std::vector<std::vector<uint32_t>> child;
        for (int e = 0; e < ne; ++e) {
            bool removed = false;
            for (int k = 0; k < R.n_lhs; ++k) removed |= slot[k] == e;
            if (!removed) child.push_back(par[e]);
        }
        for (auto& pe : prod) child.push_back(pe);
        // the kernel admits a parent to the lane path only under this neighbour-count bound
        uint32_t bound = 0, gain = 0;
        for (uint32_t v = 0; v < nvp; ++v) bound = std::max<uint32_t>(bound, pnn[v]);
        for (int k = 0; k < R.n_rhs; ++k) gain += uint32_t(R.rhs_ar[k]) * (R.rhs_ar[k] - 1u);
        if (bound + gain > 256 || nvp + R.n_fresh > 32) continue;
        // parent connectivity, and the connectivity shortcut's condition on this child: the
        // produced edges are connected and hold every vertex of the removed edges
        std::vector<uint32_t> up(nvp + R.n_fresh);
        for (uint32_t v = 0; v < up.size(); ++v) up[v] = v;
        auto root = [&](uint32_t x) { while (up[x] != x) x = up[x]; return x; };
        for (int e = 0; e < ne; ++e)
            for (int q = 1; q < pear[e]; ++q) up[root(vloc[pevo[e] + q])] = root(vloc[pevo[e]]);
        uint32_t proots = 0;
        for (uint32_t v = 0; v < nvp; ++v) proots += root(v) == v;
        const bool pconn = proots == 1;
        for (uint32_t v = 0; v < up.size(); ++v) up[v] = v;
        std::vector<bool> inp(nvp + R.n_fresh, false);
        for (int k = 0; k < R.n_rhs; ++k)
            for (int q = 0; q < R.rhs_ar[k]; ++q) {
                const uint32_t x = slot[R.n_lhs + R.rhs_off[k] + q];
                inp[x] = true;
                up[root(x)] = root(slot[R.n_lhs + R.rhs_off[k]]);
            }
        uint32_t rroots = 0;
        for (uint32_t v = 0; v < up.size(); ++v) rroots += inp[v] && root(v) == v;
        bool covers = true;
        for (int k = 0; k < R.n_lhs; ++k)
            for (int q = 0; q < pear[slot[k]]; ++q) covers = covers && inp[vloc[pevo[slot[k]] + q]];
        if (R.n_lhs > 0 && rroots == 1 && covers) R.flags |= kRuleRhsJoinsLhs;
        // per-position occurrence counts and the uniform-arity flag, as the expand kernel stages
        // them (an arity of 2..4 shared by every parent edge; the rule's RHS arity, if uniform)
        std::vector<uint32_t> pcnt(nvp, 0);
        for (int e = 0; e < ne; ++e)
            for (int q = 0; q < pear[e] && q < 4; ++q) pcnt[vloc[pevo[e] + q]] += 1u << (8 * q);
        uint32_t uni = pear[0];
        for (int e = 0; e < ne; ++e) uni = pear[e] == uni ? uni : 0u;
        if (uni < 2 || uni > 4) uni = 0;
        R.rhs_uni = R.n_rhs ? R.rhs_ar[0] : 0;
        for (int k = 0; k < R.n_rhs; ++k) R.rhs_uni = R.rhs_ar[k] == R.rhs_uni ? R.rhs_uni : 0;
        uniform += (uni && uni == R.rhs_uni) ? 1 : 0;
        const uint32_t pinfo = (pconn ? 1u : 0u) | (uni << 8);
        WlInfo info;
        const uint64_t got = lane_wl_core<32, 256>(pear.data(), pevo.data(), vloc.data(), poff.data(),
                                                   pocc.data(), pdeg.data(), pnn.data(), pnoff.data(),
                                                   pnbr.data(), pcnt.data(), pinfo, uint32_t(ne), nvp,
                                                   R, slot.data(), info);
        const uint64_t want = hgx_oracle::wl_hash(child);
        shortcut += pconn && (R.flags & kRuleRhsJoinsLhs) ? 1 : 0;
        if (got != want) {
            if (fails < 5) std::printf("trial %d: lane %016llx oracle %016llx (ne %d nvp %u)\n", t,
                                       (unsigned long long)got, (unsigned long long)want, ne, nvp);
            ++fails;
        }
    }
    std::printf("%d / %d mismatches (%d with the connectivity shortcut, %d with uniform arity)\n",
                fails, trials, shortcut, uniform);
    return fails ? 1 : 0;
}
