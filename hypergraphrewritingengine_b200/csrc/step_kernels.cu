// Kernels of one level-synchronous multiway step. See step_kernels.cuh for the stage list.
//
// Semantics restated from the reference (paths inside the reference project):
//   binding / edge-injective join   common/include/hgcommon/match_core.hpp:32-49,
//                                   common/include/hgcommon/join_core.hpp:144-208
//   rewrite (fresh vertices in ascending variable order, RHS edge order)
//                                   common/include/hgcommon/rewrite_core.hpp:53-87,
//                                   hypergraph/src/rewriter.cpp:44-82
//   WL canonical hash               common/include/hgcommon/wl_core.hpp:67-202 with the input
//                                   convention of hypergraph/include/hypergraph/wl_hash.hpp:109-243
//   causal producer of an edge      hypergraph/src/rewriter.cpp:138-191
//   branchial pairs                 hypergraph/src/causal_graph.cpp:324-350
//
// Design (not a translation of the reference's GPU tree, which is one persistent launch per
// evolution with a single-thread rewrite): every stage is a warp- or thread-granular kernel over
// the whole frontier of every evolution in the batch; warps pull frontier states from a device
// work counter so uneven state sizes balance across the 148 SMs; a state's edge record is
// staged once in shared memory and every child of it is built and hashed there, so children are
// never written to HBM unless they are new class representatives.
#include "step_kernels.cuh"
#include "lane_wl.cuh"

namespace hgx {

namespace {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <typename T>
__device__ __forceinline__ T* smp(char* base, uint32_t off) {
    return reinterpret_cast<T*>(base + off);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= static_cast<uint32_t>(d)) x += y;
    }
    return x;
}

__device__ __forceinline__ uint64_t warp_sum64(uint64_t x) {
#pragma unroll
    for (int d = 16; d; d >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, d);
    return x;
}

__device__ __forceinline__ uint32_t warp_sum32(uint32_t x) {
#pragma unroll
    for (int d = 16; d; d >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, d);
    return x;
}

__device__ __forceinline__ uint32_t warp_max32(uint32_t x) {
#pragma unroll
    for (int d = 16; d; d >>= 1) x = max(x, __shfl_xor_sync(0xFFFFFFFFu, x, d));
    return x;
}

__device__ __forceinline__ void isort64(uint64_t* a, uint32_t n) {
    for (uint32_t i = 1; i < n; ++i) {
        const uint64_t k = a[i];
        uint32_t j = i;
        while (j > 0 && a[j - 1] > k) { a[j] = a[j - 1]; --j; }
        a[j] = k;
    }
}

__device__ __forceinline__ void isort32(uint32_t* a, uint32_t n) {
    for (uint32_t i = 1; i < n; ++i) {
        const uint32_t k = a[i];
        uint32_t j = i;
        while (j > 0 && a[j - 1] > k) { a[j] = a[j - 1]; --j; }
        a[j] = k;
    }
}

// Warp-aggregated add of 1 to counter[key] for the lanes in `active`.
__device__ __forceinline__ void warp_count(unsigned long long* counter, uint32_t key, bool active) {
    const uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
    if (!active) return;
    const uint32_t peers = __match_any_sync(act, key);
    if (lane_id() == static_cast<uint32_t>(__ffs(peers) - 1))
        atomicAdd(&counter[key], static_cast<unsigned long long>(__popc(peers)));
}

// Dynamic work queue over item indices: a warp takes kWorkChunk consecutive items per atomic.
// One item per grab measured best: neighbouring items (states of one evolution) have similar
// costs, so larger grabs unbalance the tail.
constexpr uint32_t kWorkChunk = 1;
struct WarpWork {
    uint32_t base = 0, k = kWorkChunk;
    __device__ __forceinline__ uint32_t next(uint32_t* counter) {
        if (k == kWorkChunk) {
            uint32_t b = 0;
            if (lane_id() == 0) b = atomicAdd(counter, kWorkChunk);
            base = __shfl_sync(0xFFFFFFFFu, b, 0);
            k = 0;
        }
        return base + k++;
    }
};

// ------------------------------------------------------------------------------------------
// Dedup table: open addressing, linear probing, per-evolution region. Key 0 is EMPTY; a WL hash
// that is itself 0 lives in the extra slot after the region. The value is the smallest arrival
// id (event id, or a root's pseudo-event id) that produced the key: the first arrival in
// canonical order wins, whatever order the warps ran in.
// ------------------------------------------------------------------------------------------
__device__ void slot_insert(const DevPtrs& P, uint64_t base, uint64_t mask, uint64_t h,
                            uint32_t arrival) {
    if (h == 0) { atomicMin(&P.tab_vals[base + mask + 1], arrival); return; }
    uint64_t slot = smix(h) & mask;
    for (uint64_t probe = 0; probe <= mask; ++probe) {
        unsigned long long* kp = &P.tab_keys[base + slot];
        unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(kp);
        if (k == 0ull) {
            k = atomicCAS(kp, 0ull, static_cast<unsigned long long>(h));
            if (k == 0ull) k = h;
        }
        if (k == h) { atomicMin(&P.tab_vals[base + slot], arrival); return; }
        slot = (slot + 1) & mask;
    }
    atomicOr(P.err, kErrTableFull);
}

__device__ uint32_t slot_lookup(const DevPtrs& P, uint64_t base, uint64_t mask, uint64_t h) {
    if (h == 0) return P.tab_vals[base + mask + 1];
    uint64_t slot = smix(h) & mask;
    for (uint64_t probe = 0; probe <= mask; ++probe) {
        const unsigned long long k = P.tab_keys[base + slot];
        if (k == h) return P.tab_vals[base + slot];
        if (k == 0ull) return kNone;
        slot = (slot + 1) & mask;
    }
    return kNone;
}

// The evolution's state dedup table (key = WL hash, value = first arrival).
__device__ __forceinline__ void table_insert(const DevPtrs& P, const DevEvo& ev, uint64_t h,
                                             uint32_t arrival) {
    slot_insert(P, ev.table_off, ev.table_mask, h, arrival);
}
__device__ __forceinline__ uint32_t table_lookup(const DevPtrs& P, const DevEvo& ev, uint64_t h) {
    return slot_lookup(P, ev.table_off, ev.table_mask, h);
}

// ------------------------------------------------------------------------------------------
// Parent staging: the state's edge record is read once (coalesced) into shared memory, and its
// vertices are renumbered to local ids by first occurrence. WL is invariant under the local
// numbering, and the join only compares vertices for equality, so nothing downstream needs the
// global vertex ids.
// ------------------------------------------------------------------------------------------
struct Parent {
    uint32_t ne, nocc, nvp;
};

__device__ Parent load_parent(const DevPtrs& P, const Layout& L, char* sm, uint32_t sid) {
    const uint32_t lane = lane_id();
    Parent pa;
    pa.ne = P.st_ne[sid];
    pa.nocc = P.st_nocc[sid];
    pa.nvp = 0;
    if (L.XI && lane == 0) *smp<uint32_t>(sm, L.o_xready) = 0;   // no join index yet
    if (pa.ne > L.NE || pa.nocc > L.NOCC) {
        if (lane == 0) atomicOr(P.err, kErrStateTooLarge);
        __syncwarp();
        pa.ne = 0;
        pa.nocc = 0;
        return pa;
    }
    const uint32_t* rec = P.arena + P.st_off[sid];
    uint32_t* peid = smp<uint32_t>(sm, L.o_peid);
    uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint32_t* glob = smp<uint32_t>(sm, L.o_occ);    // aliases the WL occurrence list
    uint32_t* first = smp<uint32_t>(sm, L.o_deg);   // aliases the WL degrees
    const uint32_t aw = (pa.ne + 3) >> 2;
    for (uint32_t i = lane; i < pa.ne; i += 32) {
        peid[i] = rec[i];
        pear[i] = static_cast<uint8_t>((rec[pa.ne + (i >> 2)] >> ((i & 3u) * 8u)) & 0xFFu);
    }
    for (uint32_t j = lane; j < pa.nocc; j += 32) glob[j] = rec[pa.ne + aw + j];
    __syncwarp();
    uint32_t run = 0;
    bool bad = false;
    for (uint32_t b = 0; b < pa.ne; b += 32) {
        const uint32_t i = b + lane;
        const uint32_t a = i < pa.ne ? pear[i] : 0u;
        bad |= __any_sync(0xFFFFFFFFu, i < pa.ne && (a == 0u || a > static_cast<uint32_t>(kMaxArity)));
        const uint32_t inc = warp_incl_scan(a);
        if (i < pa.ne) pevo[i] = static_cast<uint16_t>(run + inc - a);
        run += __shfl_sync(0xFFFFFFFFu, inc, 31);
    }
    // A record whose arities are out of range or do not add up to its occurrence count (possible
    // only for records a caller supplies; the engine writes consistent ones) would send the vertex
    // offsets past the staged occurrences: flag it and treat the state as empty.
    if (bad || run != pa.nocc) {
        if (lane == 0) atomicOr(P.err, kErrStateTooLarge);
        __syncwarp();
        pa.ne = 0;
        pa.nocc = 0;
        return pa;
    }
    if (pa.nocc > kHashOccMin && L.VT) {
        // Large state: vertex -> local id through a shared-memory hash table, O(occurrences).
        // Ids follow slot order; any consistent numbering works (WL is label-invariant and the
        // join only compares vertices for equality).
        uint32_t* tab = smp<uint32_t>(sm, L.o_vtab);
        uint16_t* tid = smp<uint16_t>(sm, L.o_vtid);
        const uint32_t TS = L.VT;
        for (uint32_t t = lane; t < TS; t += 32) tab[t] = kNone;
        __syncwarp();
        bool full = false;   // a vertex found no slot: more distinct vertices than the layout holds
        for (uint32_t j = lane; j < pa.nocc; j += 32) {
            const uint32_t v = glob[j];
            uint32_t h = (v * 2654435761u) & (TS - 1);
            bool placed = false;
            for (uint32_t probe = 0; probe < TS; ++probe) {
                const uint32_t prev = atomicCAS(&tab[h], kNone, v);
                if (prev == kNone || prev == v) { placed = true; break; }
                h = (h + 1) & (TS - 1);
            }
            full |= !placed;
            first[j] = h;
        }
        if (__any_sync(0xFFFFFFFFu, full)) {
            if (lane == 0) atomicOr(P.err, kErrStateTooLarge);
            __syncwarp();
            pa.ne = 0;
            pa.nocc = 0;
            return pa;
        }
        __syncwarp();
        uint32_t ids = 0;
        for (uint32_t b = 0; b < TS; b += 32) {
            const uint32_t t = b + lane;
            const bool used = tab[t] != kNone;
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, used);
            if (used) tid[t] = static_cast<uint16_t>(ids + __popc(bal & ((1u << lane) - 1u)));
            ids += __popc(bal);
        }
        __syncwarp();
        for (uint32_t j = lane; j < pa.nocc; j += 32) vloc[j] = tid[first[j]];
        __syncwarp();
        pa.nvp = ids;
        if (ids > L.NV) {   // more vertices than the layout's per-vertex arrays hold
            if (lane == 0) atomicOr(P.err, kErrStateTooLarge);
            __syncwarp();
            pa.ne = pa.nocc = pa.nvp = 0;
        }
        return pa;
    }
    run = 0;
    for (uint32_t b = 0; b < pa.nocc; b += 32) {
        const uint32_t j = b + lane;
        uint32_t f = j;
        if (j < pa.nocc) {
            const uint32_t v = glob[j];
            for (uint32_t i = 0; i < j; ++i)
                if (glob[i] == v) { f = i; break; }
            first[j] = f;
        }
        const bool rep = (j < pa.nocc) && f == j;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, rep);
        if (rep) vloc[j] = static_cast<uint16_t>(run + __popc(bal & ((1u << lane) - 1u)));
        run += __popc(bal);
    }
    __syncwarp();
    for (uint32_t j = lane; j < pa.nocc; j += 32) {
        const uint32_t f = first[j];
        if (f != j) vloc[j] = vloc[f];
    }
    __syncwarp();
    pa.nvp = run;
    if (run > L.NV) {   // more vertices than the layout's per-vertex arrays hold
        if (lane == 0) atomicOr(P.err, kErrStateTooLarge);
        __syncwarp();
        pa.ne = pa.nocc = pa.nvp = 0;
    }
    return pa;
}

__device__ __forceinline__ void load_rule(char* sm, const Layout& L, const DevRule* src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = smp<uint32_t>(sm, L.o_rule);
    for (uint32_t i = lane_id(); i < sizeof(DevRule) / 4; i += 32) d[i] = s[i];
    __syncwarp();
}

// ------------------------------------------------------------------------------------------
// Join indices of a staged state of more than kJoinIndexMin edges, built once per staging in the
// warp's shared memory and used by every join over the state (all rules, all slices):
//   * vertex index (the reference's InvertedVertexIndex, hypergraph/include/hypergraph/
//     index.hpp:134-230): per local vertex, the state positions of the edges holding it, each
//     edge once. A pattern edge with a bound variable draws its candidates from the bound vertex
//     of smallest degree instead of from every edge.
//   * signature index (SignatureIndex, index.hpp:30-130; signatures as in common/include/
//     hgcommon/signature_core.hpp:24-84): the edges bucketed by arity and vertex-repetition
//     pattern (nibble q = the first position holding the same vertex as position q). A pattern
//     edge with no bound variable draws its candidates from the buckets whose edges repeat a
//     vertex wherever the pattern repeats a variable. Built only when the state's edges fall in
//     at most kSigBuckets signatures; edges of arity 16 share one bucket that is always searched.
// Every candidate still passes the full test, so the indices only skip edges that would fail it.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t edge_signature(const uint16_t* v, uint32_t a) {
    if (a >= 16) return ~1ull;                 // the unindexed bucket
    uint64_t code = uint64_t(a) << 60;
    for (uint32_t q = 1; q < a; ++q) {
        uint32_t r = 0;
        while (v[r] != v[q]) ++r;              // r <= q
        code |= uint64_t(r) << (4 * q);
    }
    return code;
}

// Pattern edge (arity a, variables pv) against a bucket key: equal arity, and every position
// whose variable repeats an earlier one holds the same vertex there.
__device__ __forceinline__ bool signature_compatible(const uint8_t* pv, uint32_t a, uint64_t key) {
    if (key == ~1ull) return a >= 16;
    if ((key >> 60) != a) return false;
    for (uint32_t q = 1; q < a; ++q) {
        uint32_t r = 0;
        while (pv[r] != pv[q]) ++r;
        if (r != q && ((key >> (4 * q)) & 15u) != ((key >> (4 * r)) & 15u)) return false;
    }
    return true;
}

__device__ void build_join_index(const Layout& L, char* sm, const Parent& pa) {
    if (!L.XI || pa.ne <= kJoinIndexMin) return;
    const uint32_t lane = lane_id();
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint32_t* xoff = smp<uint32_t>(sm, L.o_xoff);
    uint16_t* xinc = smp<uint16_t>(sm, L.o_xinc);
    uint64_t* bkey = smp<uint64_t>(sm, L.o_bkey);
    uint32_t* boff = smp<uint32_t>(sm, L.o_boff);
    uint16_t* blist = smp<uint16_t>(sm, L.o_blist);
    uint32_t* misc = smp<uint32_t>(sm, L.o_misc);   // [0] bucket count (kSigBuckets+1 = overflow)
    // vertex index: degrees (an edge counts once per distinct vertex), scan, fill
    for (uint32_t v = lane; v <= pa.nvp; v += 32) xoff[v] = 0;
    if (lane == 0) misc[0] = 0;
    __syncwarp();
    for (uint32_t e = lane; e < pa.ne; e += 32) {
        const uint32_t a = pear[e], vo = pevo[e];
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t v = vloc[vo + q];
            bool first = true;
            for (uint32_t r = 0; r < q && first; ++r) first = vloc[vo + r] != v;
            if (first) atomicAdd(&xoff[v + 1], 1u);
        }
    }
    __syncwarp();
    uint32_t run = 0;
    for (uint32_t b = 0; b <= pa.nvp; b += 32) {
        const uint32_t i = b + lane;
        const uint32_t c = i <= pa.nvp ? xoff[i] : 0u;
        const uint32_t inc = warp_incl_scan(c);
        __syncwarp();
        if (i <= pa.nvp) xoff[i] = run + inc;   // xoff[v + 1] = end of v's list
        run += __shfl_sync(0xFFFFFFFFu, inc, 31);
        __syncwarp();
    }
    // fill from each list's end backwards (the order inside a list does not matter: candidates
    // are collected into a bitmask over state positions)
    for (uint32_t e = lane; e < pa.ne; e += 32) {
        const uint32_t a = pear[e], vo = pevo[e];
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t v = vloc[vo + q];
            bool first = true;
            for (uint32_t r = 0; r < q && first; ++r) first = vloc[vo + r] != v;
            if (first) xinc[atomicSub(&xoff[v + 1], 1u) - 1u] = static_cast<uint16_t>(e);
        }
    }
    __syncwarp();
    // xoff[v + 1] now holds the start of v's list: shift back (xoff[nvp] = total)
    for (uint32_t b = 0; b <= pa.nvp; b += 32) {
        const uint32_t i = b + lane;
        const uint32_t x = i + 1 <= pa.nvp ? xoff[i + 1] : run;
        __syncwarp();
        if (i <= pa.nvp) xoff[i] = i == 0 ? 0u : x;
        __syncwarp();
    }
    // signature index: the distinct keys of each 32-edge chunk (match_any), appended to the
    // bucket list one leader at a time; more than kSigBuckets keys leaves it unbuilt
    for (uint32_t b = 0; b < pa.ne && misc[0] <= kSigBuckets; b += 32) {
        const uint32_t e = b + lane;
        const uint64_t key = e < pa.ne ? edge_signature(&vloc[pevo[e]], pear[e]) : ~0ull;
        const uint32_t grp = __match_any_sync(0xFFFFFFFFu, key);
        uint32_t leaders = __ballot_sync(0xFFFFFFFFu, e < pa.ne && (__ffs(grp) - 1) == static_cast<int>(lane));
        while (leaders) {
            const int l = __ffs(leaders) - 1;
            leaders &= leaders - 1;
            const uint64_t k = __shfl_sync(0xFFFFFFFFu, key, l);
            const uint32_t nb = misc[0];
            const bool hit = lane < min(nb, kSigBuckets) && bkey[lane] == k;
            if (!__any_sync(0xFFFFFFFFu, hit) && lane == 0 && nb <= kSigBuckets) {
                if (nb < kSigBuckets) bkey[nb] = k;
                misc[0] = nb + 1;
            }
            __syncwarp();
        }
    }
    const uint32_t nb = misc[0];
    const bool sig = nb <= kSigBuckets;
    if (sig) {
        // bucket sizes, offsets, then the lists (each edge into its bucket)
        for (uint32_t k = lane; k <= nb; k += 32) boff[k] = 0;
        __syncwarp();
        for (uint32_t e = lane; e < pa.ne; e += 32) {
            const uint64_t key = edge_signature(&vloc[pevo[e]], pear[e]);
            uint32_t k = 0;
            while (k < nb && bkey[k] != key) ++k;
            atomicAdd(&boff[k + 1], 1u);
        }
        __syncwarp();
        if (lane == 0)
            for (uint32_t k = 1; k <= nb; ++k) boff[k] += boff[k - 1];
        __syncwarp();
        for (uint32_t e = lane; e < pa.ne; e += 32) {
            const uint64_t key = edge_signature(&vloc[pevo[e]], pear[e]);
            uint32_t k = 0;
            while (k < nb && bkey[k] != key) ++k;
            blist[atomicSub(&boff[k + 1], 1u) - 1u] = static_cast<uint16_t>(e);
        }
        __syncwarp();
        // boff[k + 1] now holds the start of bucket k: shift back
        if (lane == 0) {
            for (uint32_t k = 0; k < nb; ++k) boff[k] = boff[k + 1];
            boff[nb] = pa.ne;
        }
    }
    if (lane == 0) *smp<uint32_t>(sm, L.o_xready) = 1u | (sig ? 2u : 0u) | (nb << 8);
    __syncwarp();
}

// ------------------------------------------------------------------------------------------
// The join. One warp holds one partial match; at every depth the 32 lanes test the state's
// edges against the next pattern edge in parallel and a ballot compacts the survivors into a
// candidate bitmask. Candidates are taken in ascending state position, so matches come out in
// lexicographic order of their positions in schedule order -- the canonical event order.
// Edge-injective (a state edge serves one pattern edge), vertex-non-injective.
// ------------------------------------------------------------------------------------------
__device__ void compute_cands(const Layout& L, char* sm, const DevRule& R, uint32_t p,
                              const Parent& pa, uint32_t mask, uint32_t* cand) {
    const uint32_t lane = lane_id();
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    const uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
    const uint32_t* taken = smp<uint32_t>(sm, L.o_taken);
    const uint32_t a = R.lhs_ar[p];
    const uint8_t* pv = &R.lhs_vars[R.lhs_off[p]];
    // state edge i can take pattern edge p under the current binding
    auto ok_at = [&](uint32_t i) -> bool {
        if (pear[i] != a || ((taken[i >> 5] >> (i & 31u)) & 1u)) return false;
        const uint32_t vo = pevo[i];
        bool ok = true;
        for (uint32_t q = 0; q < a && ok; ++q) {
            const uint32_t var = pv[q];
            const uint32_t x = vloc[vo + q];
            if ((mask >> var) & 1u) {
                ok = (bind[var] == x);
            } else {
                for (uint32_t r = 0; r < q; ++r)
                    if (pv[r] == var) { ok = (vloc[vo + r] == x); break; }
            }
        }
        return ok;
    };
    const uint32_t xr = L.XI ? *smp<uint32_t>(sm, L.o_xready) : 0u;
    if (xr) {
        // indexed candidates: the edges of the bound vertex of smallest degree, else the edges of
        // the signature buckets compatible with the pattern edge
        const uint32_t* xoff = smp<uint32_t>(sm, L.o_xoff);
        uint32_t best = 0xFFFFFFFFu, bx = 0;
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t var = pv[q];
            if (!((mask >> var) & 1u)) continue;
            const uint32_t x = bind[var];
            const uint32_t deg = xoff[x + 1] - xoff[x];
            if (deg < best) { best = deg; bx = x; }
        }
        const bool use_v = best != 0xFFFFFFFFu;
        if (use_v || (xr & 2u)) {
            const uint32_t nw = (pa.ne + 31) >> 5;
            for (uint32_t w = lane; w < nw; w += 32) cand[w] = 0;
            __syncwarp();
            if (use_v) {
                const uint16_t* list = smp<uint16_t>(sm, L.o_xinc) + xoff[bx];
                for (uint32_t j = lane; j < best; j += 32) {
                    const uint32_t i = list[j];
                    if (ok_at(i)) atomicOr(&cand[i >> 5], 1u << (i & 31u));
                }
            } else {
                const uint64_t* bkey = smp<uint64_t>(sm, L.o_bkey);
                const uint32_t* boff = smp<uint32_t>(sm, L.o_boff);
                const uint16_t* blist = smp<uint16_t>(sm, L.o_blist);
                const uint32_t nb = xr >> 8;
                for (uint32_t k = 0; k < nb; ++k) {
                    if (!signature_compatible(pv, a, bkey[k])) continue;
                    for (uint32_t j = boff[k] + lane; j < boff[k + 1]; j += 32) {
                        const uint32_t i = blist[j];
                        if (ok_at(i)) atomicOr(&cand[i >> 5], 1u << (i & 31u));
                    }
                }
            }
            __syncwarp();
            return;
        }
    }
    for (uint32_t b = 0; b < pa.ne; b += 32) {
        const uint32_t i = b + lane;
        const bool ok = i < pa.ne && ok_at(i);
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, ok);
        if (lane == 0) cand[b >> 5] = bal;
    }
    __syncwarp();
}

// Skipping in the warp join: at the last pattern position every candidate is one match, so a
// caller that does not need a run of leading matches (a slice that starts past them, or a
// count) takes the whole candidate set at once -- its popcount -- instead of walking it. The
// policy says how many leading matches the caller still wants skipped (left) and learns how many
// were (take); `want` and the counter are warp-uniform.
struct NoSkip {
    __device__ uint32_t left() const { return 0u; }
    __device__ void take(uint32_t) const {}
};
struct SkipCounter {
    uint32_t* n;     // matches passed so far (enumerated or skipped)
    uint32_t want;   // skip while fewer than this have passed
    __device__ uint32_t left() const { return want > *n ? want - *n : 0u; }
    __device__ void take(uint32_t c) const { *n += c; }
};

// sched: the binding order of the LHS positions; seed >= 0 pins the first scheduled position to
// that state position (a seeded join: every emitted match uses it there). limit: stop once this
// many matches have passed (enumerated or skipped).
template <class F, class Skip = NoSkip>
__device__ void warp_join(const Layout& L, char* sm, const DevRule& R, const Parent& pa,
                          const uint8_t* sched, int seed, F&& on_match,
                          uint32_t limit = 0xFFFFFFFFu, Skip skip = Skip()) {
    const uint32_t lane = lane_id();
    const uint32_t n = R.n_lhs;
    const uint32_t nw = (pa.ne + 31) >> 5;
    if (n == 0 || pa.ne == 0) return;
    uint32_t* cand = smp<uint32_t>(sm, L.o_cand);
    uint32_t* taken = smp<uint32_t>(sm, L.o_taken);
    uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
    uint16_t* match = smp<uint16_t>(sm, L.o_match);
    uint16_t* mdepth = smp<uint16_t>(sm, L.o_mdepth);
    uint32_t* saved = smp<uint32_t>(sm, L.o_misc);
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    (void)pear;
    for (uint32_t w = lane; w < nw; w += 32) taken[w] = 0;
    __syncwarp();
    uint32_t mask = 0;
    uint32_t d = 0;
    // the candidates of the last position at depth dd, taken whole when the caller skips them all
    auto try_skip = [&](uint32_t dd) {
        const uint32_t want = skip.left();
        if (!want) return;
        uint32_t c = 0;
        for (uint32_t w = lane; w < nw; w += 32) c += __popc(cand[dd * L.W + w]);
        c = warp_sum32(c);
        if (c == 0 || c > want) return;
        skip.take(c);
        limit -= c;
        for (uint32_t w = lane; w < nw; w += 32) cand[dd * L.W + w] = 0;
        __syncwarp();
    };
    compute_cands(L, sm, R, sched[0], pa, mask, cand);
    if (seed >= 0) {
        // keep only the seed among the first position's candidates
        for (uint32_t w = lane; w < nw; w += 32)
            cand[w] &= (static_cast<uint32_t>(seed) >> 5) == w ? (1u << (seed & 31)) : 0u;
        __syncwarp();
    }
    if (n == 1) try_skip(0);
    while (true) {
        int pick = -1;
        for (uint32_t w = 0; w < nw; ++w) {
            const uint32_t c = cand[d * L.W + w];
            if (c) { pick = static_cast<int>(w * 32 + __ffs(c) - 1); break; }
        }
        __syncwarp();
        if (pick < 0) {
            if (d == 0) break;
            --d;
            const uint32_t e = mdepth[d];
            mask = saved[d];
            __syncwarp();
            if (lane == 0) taken[e >> 5] &= ~(1u << (e & 31u));
            __syncwarp();
            continue;
        }
        const uint32_t p = sched[d];
        if (lane == 0) {
            cand[d * L.W + (pick >> 5)] &= ~(1u << (pick & 31));
            taken[pick >> 5] |= 1u << (pick & 31);
            match[p] = static_cast<uint16_t>(pick);
            mdepth[d] = static_cast<uint16_t>(pick);
            saved[d] = mask;
        }
        const uint32_t a = R.lhs_ar[p];
        const uint8_t* pv = &R.lhs_vars[R.lhs_off[p]];
        const uint32_t vo = pevo[pick];
        uint32_t nm = mask;
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t var = pv[q];
            if (!((nm >> var) & 1u)) {
                if (lane == 0) bind[var] = vloc[vo + q];
                nm |= 1u << var;
            }
        }
        __syncwarp();
        if (d + 1 == n) {
            on_match(nm);
            __syncwarp();
            if (lane == 0) taken[pick >> 5] &= ~(1u << (pick & 31));
            __syncwarp();
            if (--limit == 0) break;   // the caller needs no later match
        } else {
            mask = nm;
            ++d;
            compute_cands(L, sm, R, sched[d], pa, mask, cand + d * L.W);
            if (d + 1 == n) try_skip(d);
        }
    }
    __syncwarp();
}

// ------------------------------------------------------------------------------------------
// Lane-parallel join for small staged states (<= 64 edges, <= kLaneJoinLhs LHS edges). Lane i
// takes state edge e0 at the first scheduled position and walks the remaining positions on its
// own, depth first, edges ascending; no warp synchronisation inside the walk. A lane's matches
// come out in the lexicographic order of their state positions taken in schedule order -- the
// order warp_join enumerates -- and lanes hold ascending e0, so (e0, walk order) is the canonical
// match order. on_match(packed) receives the pattern-order positions, one byte each.
// ------------------------------------------------------------------------------------------
template <class F>
__device__ uint32_t lane_walk(const Layout& L, const char* sm, const DevRule& R, const Parent& pa,
                              uint32_t e0, F&& on_match, uint32_t j1_lo = 0,
                              uint32_t j1_hi = 0xFFFFFFFFu) {
    const uint8_t* pear = smp<uint8_t>(const_cast<char*>(sm), L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(const_cast<char*>(sm), L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(const_cast<char*>(sm), L.o_vloc);
    const uint32_t n = R.n_lhs;
    if (n == 2) {
        // two pattern edges: bind the first at e0, then every second edge in ascending order
        // (the same matches in the same order as the depth-first walk below)
        const uint32_t p0 = R.sched[0], p1 = R.sched[1];
        const uint32_t a0 = R.lhs_ar[p0], a1 = R.lhs_ar[p1];
        if (pear[e0] != a0) return 0;
        uint16_t bind[kMaxVars];
        uint32_t bound = 0;
        const uint8_t* v0 = &R.lhs_vars[R.lhs_off[p0]];
        const uint8_t* v1 = &R.lhs_vars[R.lhs_off[p1]];
        const uint32_t vo0 = pevo[e0];
        for (uint32_t q = 0; q < a0; ++q) {
            const uint32_t var = v0[q];
            const uint16_t x = vloc[vo0 + q];
            if ((bound >> var) & 1u) {
                if (bind[var] != x) return 0;
            } else {
                bind[var] = x;
                bound |= 1u << var;
            }
        }
        uint32_t found = 0;
        const uint32_t jend = min(pa.ne, j1_hi);
        for (uint32_t j = j1_lo; j < jend; ++j) {
            if (j == e0 || pear[j] != a1) continue;
            const uint32_t vo = pevo[j];
            uint32_t nb = 0;
            bool ok = true;
            for (uint32_t q = 0; q < a1 && ok; ++q) {
                const uint32_t var = v1[q];
                const uint16_t x = vloc[vo + q];
                if (((bound | nb) >> var) & 1u) {
                    ok = bind[var] == x;
                } else {
                    bind[var] = x;
                    nb |= 1u << var;
                }
            }
            if (!ok) continue;
            on_match((e0 << (8u * p0)) | (j << (8u * p1)));
            ++found;
        }
        return found;
    }
    uint16_t bind[kMaxVars];
    uint32_t bound = 0;
    uint32_t newly[kLaneJoinLhs];
    uint32_t pick[kLaneJoinLhs];
    uint64_t used = 0;
    // bind pattern position sched[d] to state edge j; on failure nothing stays bound
    auto try_bind = [&](uint32_t d, uint32_t j) -> bool {
        const uint32_t p = R.sched[d];
        const uint32_t a = R.lhs_ar[p];
        if (pear[j] != a) return false;
        const uint8_t* pv = &R.lhs_vars[R.lhs_off[p]];
        const uint32_t vo = pevo[j];
        uint32_t nb = 0;
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t var = pv[q];
            const uint16_t x = vloc[vo + q];
            if ((bound >> var) & 1u) {
                if (bind[var] != x) { bound &= ~nb; return false; }
            } else {
                bind[var] = x;
                bound |= 1u << var;
                nb |= 1u << var;
            }
        }
        newly[d] = nb;
        return true;
    };
    if (!try_bind(0, e0)) return 0;
    pick[0] = e0;
    used = 1ull << e0;
    uint32_t found = 0;
    uint32_t d = 1, j = 0;
    while (d > 0) {
        if (d == n) {
            uint32_t packed = 0;
            for (uint32_t k = 0; k < n; ++k) packed |= pick[k] << (8u * R.sched[k]);
            on_match(packed);
            ++found;
            --d;
            if (d == 0) break;
            bound &= ~newly[d];
            used &= ~(1ull << pick[d]);
            j = pick[d] + 1;
            continue;
        }
        bool ok = false;
        const uint32_t jend = d == 1 ? min(pa.ne, j1_hi) : pa.ne;
        if (d == 1 && j < j1_lo) j = j1_lo;
        for (; j < jend; ++j)
            if (!((used >> j) & 1ull) && try_bind(d, j)) { ok = true; break; }
        if (ok) {
            pick[d] = j;
            used |= 1ull << j;
            ++d;
            j = 0;
        } else {
            --d;
            if (d == 0) break;
            bound &= ~newly[d];
            used &= ~(1ull << pick[d]);
            j = pick[d] + 1;
        }
    }
    return found;
}

// Matches of (state, rule) by lane walks over every first edge, warp total. A state of at most 16
// (8) edges gives each first edge 2 (4) lanes, which split the second position's candidates.
__device__ uint32_t lane_join_count(const Layout& L, const char* sm, const DevRule& R,
                                    const Parent& pa) {
    uint32_t c = 0;
    const uint32_t lane = lane_id();
    const uint32_t parts = (R.n_lhs < 2 || pa.ne > 16) ? 1u : (pa.ne <= 8 ? 4u : 2u);
    if (parts > 1) {
        const uint32_t e0 = lane / parts, part = lane % parts;
        const uint32_t span = (pa.ne + parts - 1) / parts;
        if (e0 < pa.ne)
            c = lane_walk(L, sm, R, pa, e0, [](uint32_t) {}, part * span, (part + 1) * span);
        return warp_sum32(c);
    }
    for (uint32_t b = 0; b < pa.ne; b += 32)
        if (b + lane < pa.ne) c += lane_walk(L, sm, R, pa, b + lane, [](uint32_t) {});
    return warp_sum32(c);
}

// ------------------------------------------------------------------------------------------
// Child construction in shared memory: parent edges minus the matched ones (ascending, so the
// reference's ascending edge-id order is kept) followed by the produced edges in RHS order.
// Vertices stay local: a matched variable takes its bound local id, the n-th fresh variable
// takes local id nvp + n.
// ------------------------------------------------------------------------------------------
__device__ uint32_t build_child(const Layout& L, char* sm, const DevRule& R, const Parent& pa,
                                uint32_t nm) {
    const uint32_t lane = lane_id();
    const uint32_t* taken = smp<uint32_t>(sm, L.o_taken);
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    const uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
    uint8_t* car = smp<uint8_t>(sm, L.o_car);
    uint16_t* cvo = smp<uint16_t>(sm, L.o_cvo);
    uint32_t run = 0;
    for (uint32_t b = 0; b < pa.ne; b += 32) {
        const uint32_t i = b + lane;
        const bool keep = i < pa.ne && !((taken[i >> 5] >> (i & 31u)) & 1u);
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
        if (keep) {
            const uint32_t c = run + __popc(bal & ((1u << lane) - 1u));
            car[c] = pear[i];
            cvo[c] = pevo[i];
        }
        run += __popc(bal);
    }
    for (uint32_t k = lane; k < R.n_rhs; k += 32) {
        car[run + k] = R.rhs_ar[k];
        cvo[run + k] = static_cast<uint16_t>(pa.nocc + R.rhs_off[k]);
    }
    for (uint32_t t = lane; t < R.rhs_total; t += 32) {
        const uint32_t var = R.rhs_vars[t];
        vloc[pa.nocc + t] = ((nm >> var) & 1u) ? bind[var]
                                                : static_cast<uint16_t>(pa.nvp + R.fresh_rank[var]);
    }
    __syncwarp();
    return run + R.n_rhs;
}

// ------------------------------------------------------------------------------------------
// WL canonical hash of the state held in shared memory (car/cvo/vloc, `ne` edges over local
// vertex ids [0, V)), computed by one warp: lanes own vertices. Bit-identical to the reference
// core: initial colour FNV(deg, sorted (arity,pos) of the first `cap` occurrences), rounds of
// sorted neighbour folds until the distinct-colour count stops changing (<= 100), then the
// component fold and the final FNV over (n_v, n_e, sums).
// ------------------------------------------------------------------------------------------
__device__ uint32_t wl_distinct(const uint64_t* cur, const uint32_t* deg, uint32_t V, uint32_t nv,
                                uint64_t* srt) {
    const uint32_t lane = lane_id();
    if (V <= 32) {
        // one vertex per lane: equal colours found by match_any among the present lanes
        const bool present = lane < V && deg[lane] != 0;
        const uint32_t pm = __ballot_sync(0xFFFFFFFFu, present);
        bool lead = false;
        if (present) {
            const uint32_t grp = __match_any_sync(pm, static_cast<unsigned long long>(cur[lane]));
            lead = lane == static_cast<uint32_t>(__ffs(grp) - 1);
        }
        return __popc(__ballot_sync(0xFFFFFFFFu, lead));
    }
    // a shared-memory hash set of the present colours (>= 2 slots per vertex, linear probing,
    // key 0 = empty; colour 0 itself is a flag in the slot after the table): every first insert
    // of a colour counts once
    (void)nv;
    uint32_t n2 = 64;
    while (n2 < 2 * V) n2 <<= 1;
    for (uint32_t i = lane; i <= n2; i += 32) srt[i] = 0;
    __syncwarp();
    uint32_t d = 0;
    for (uint32_t v = lane; v < V; v += 32) {
        if (!deg[v]) continue;
        const unsigned long long c = cur[v];
        if (c == 0) {
            d += atomicExch(reinterpret_cast<unsigned long long*>(&srt[n2]), 1ull) == 0 ? 1u : 0u;
            continue;
        }
        uint32_t slot = static_cast<uint32_t>(smix(c)) & (n2 - 1);
        for (uint32_t probe = 0; probe < n2; ++probe) {
            const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(&srt[slot]), 0ull, c);
            if (old == 0) { ++d; break; }
            if (old == c) break;
            slot = (slot + 1) & (n2 - 1);
        }
    }
    const uint32_t total = warp_sum32(d);
    __syncwarp();
    return total;
}

// Whether a staged parent is one component: lock-free union-find over its edges (as in warp_wl),
// then one root among its vertices (every staged vertex occurs in an edge). Uses the layout's
// component scratch.
__device__ bool parent_connected(const Layout& L, char* sm, const Parent& pa) {
    const uint32_t lane = lane_id();
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint32_t* comp = smp<uint32_t>(sm, L.o_comp);
    for (uint32_t v = lane; v < pa.nvp; v += 32) comp[v] = v;
    __syncwarp();
    {
        volatile uint32_t* vc = comp;
        for (uint32_t e = lane; e < pa.ne; e += 32) {
            const uint32_t a = pear[e], vo = pevo[e];
            for (uint32_t q = 1; q < a; ++q) {
                uint32_t x = vloc[vo], y = vloc[vo + q];
                for (uint32_t tries = 0; tries < 2 * pa.nvp + 8; ++tries) {
                    while (vc[x] != x) x = vc[x];
                    while (vc[y] != y) y = vc[y];
                    if (x == y) break;
                    if (x < y) { const uint32_t t = x; x = y; y = t; }
                    if (atomicCAS(&comp[x], x, y) == x) break;
                }
            }
        }
    }
    __syncwarp();
    uint32_t nroots = 0;
    for (uint32_t v = lane; v < pa.nvp; v += 32) nroots += comp[v] == v ? 1u : 0u;
    const bool one = warp_sum32(nroots) == 1;
    __syncwarp();
    return one;
}

// connected: the child is known to be one component (a connected parent under a rule whose
// right-hand side joins every left-hand vertex): the union-find is skipped.
__device__ uint64_t warp_wl(const Layout& L, char* sm, uint32_t ne, uint32_t V, WlInfo& info,
                        bool connected = false) {
    const uint32_t lane = lane_id();
    const uint8_t* car = smp<uint8_t>(sm, L.o_car);
    const uint16_t* cvo = smp<uint16_t>(sm, L.o_cvo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint64_t* cur = smp<uint64_t>(sm, L.o_cur);
    uint64_t* nxt = smp<uint64_t>(sm, L.o_nxt);
    uint64_t* csum = smp<uint64_t>(sm, L.o_csum);
    uint64_t* ccnt = smp<uint64_t>(sm, L.o_ccnt);
    uint64_t* nbr = smp<uint64_t>(sm, L.o_nbr);
    uint32_t* occ = smp<uint32_t>(sm, L.o_occ);
    uint32_t* ooff = smp<uint32_t>(sm, L.o_ooff);
    uint32_t* nbo = smp<uint32_t>(sm, L.o_nbo);
    uint32_t* deg = smp<uint32_t>(sm, L.o_deg);
    uint32_t* nn = smp<uint32_t>(sm, L.o_nn);
    uint32_t* comp = smp<uint32_t>(sm, L.o_comp);

    info.rounds = 0;
    info.nv = 0;
    info.nocc = 0;
    info.nbr = 0;
    if (ne == 0) return kEmptyStateHash;

    for (uint32_t v = lane; v < V; v += 32) { deg[v] = 0; nn[v] = 0; }
    __syncwarp();
    for (uint32_t e = lane; e < ne; e += 32) {
        const uint32_t a = car[e], vo = cvo[e];
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t v = vloc[vo + q];
            atomicAdd(&deg[v], 1u);
            atomicAdd(&nn[v], a - 1u);
        }
    }
    __syncwarp();
    uint32_t run_o = 0, run_n = 0, run_nn = 0, nv = 0, cap = 1;
    for (uint32_t b = 0; b < V; b += 32) {
        const uint32_t v = b + lane;
        const uint32_t dv = v < V ? deg[v] : 0u;
        const uint32_t nnv = v < V ? nn[v] : 0u;
        const uint32_t s = max(nnv, dv);
        const uint32_t io = warp_incl_scan(dv);
        const uint32_t is = warp_incl_scan(s);
        if (v < V) {
            ooff[v] = run_o + io - dv;
            nbo[v] = run_n + is - s;
            comp[v] = run_o + io - dv;
        }
        run_o += __shfl_sync(0xFFFFFFFFu, io, 31);
        run_n += __shfl_sync(0xFFFFFFFFu, is, 31);
        nv += __popc(__ballot_sync(0xFFFFFFFFu, dv > 0));
        cap = max(cap, warp_max32(nnv));
        run_nn += warp_sum32(nnv);
    }
    info.nv = nv;
    info.nocc = run_o;
    info.nbr = run_nn;   // sum over edges of a(a-1): neighbour entries per refinement round
    if (nv == 0) return 0;   // only arity-0 edges: the reference core returns 0
    __syncwarp();
    for (uint32_t e = lane; e < ne; e += 32) {
        const uint32_t a = car[e], vo = cvo[e];
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t slot = atomicAdd(&comp[vloc[vo + q]], 1u);
            occ[slot] = (e << 8) | q;
        }
    }
    __syncwarp();

    // initial colours
    for (uint32_t v = lane; v < V; v += 32) {
        const uint32_t dv = deg[v];
        if (!dv) continue;
        uint32_t* o = occ + ooff[v];
        if (dv > cap) isort32(o, dv);   // truncation keeps the first `cap` in edge order
        uint64_t* kb = nbr + nbo[v];
        const uint32_t n = min(dv, cap);
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t x = o[j];
            kb[j] = (static_cast<uint64_t>(car[x >> 8]) << 8) | (x & 0xFFu);
        }
        isort64(kb, n);
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(dv));
        for (uint32_t j = 0; j < n; ++j) {
            h = fnv(h, kb[j] >> 8);
            h = fnv(h, kb[j] & 0xFFu);
        }
        cur[v] = h;
    }
    __syncwarp();
    uint64_t* srt = smp<uint64_t>(sm, L.o_srt);
    uint32_t prev = wl_distinct(cur, deg, V, nv, srt);
    for (uint32_t it = 0; it < kWlMaxRounds; ++it) {
        for (uint32_t v = lane; v < V; v += 32) {
            const uint32_t dv = deg[v];
            if (!dv) continue;
            const uint32_t* o = occ + ooff[v];
            uint64_t* kb = nbr + nbo[v];
            uint32_t n = 0;
            for (uint32_t j = 0; j < dv; ++j) {
                const uint32_t x = o[j];
                const uint32_t e = x >> 8, q = x & 0xFFu;
                const uint32_t a = car[e], vo = cvo[e];
                for (uint32_t k = 0; k < a; ++k)
                    if (k != q && n < cap) kb[n++] = fnv(cur[vloc[vo + k]], k);
            }
            isort64(kb, n);
            uint64_t h = cur[v];
            for (uint32_t j = 0; j < n; ++j) h = fnv(h, kb[j]);
            nxt[v] = h;
        }
        __syncwarp();
        for (uint32_t v = lane; v < V; v += 32) cur[v] = nxt[v];
        __syncwarp();
        const uint32_t dd = wl_distinct(cur, deg, V, nv, srt);
        ++info.rounds;
        if (dd == prev) break;
        prev = dd;
    }

    // components (union-find on one lane; the partition is what enters the hash)
    bool one = connected;
    if (!connected) {
        for (uint32_t v = lane; v < V; v += 32) { comp[v] = v; csum[v] = 0; ccnt[v] = 0; }
        __syncwarp();
        // lock-free union-find: a root is only ever hooked under a smaller root (atomicCAS), so the
        // forest stays acyclic and every failed hook means another lane made progress
        {
            volatile uint32_t* vc = comp;
            for (uint32_t e = lane; e < ne; e += 32) {
                const uint32_t a = car[e], vo = cvo[e];
                for (uint32_t q = 1; q < a; ++q) {
                    uint32_t x = vloc[vo], y = vloc[vo + q];
                    for (uint32_t tries = 0; tries < 2 * V + 8; ++tries) {
                        while (vc[x] != x) x = vc[x];
                        while (vc[y] != y) y = vc[y];
                        if (x == y) break;
                        if (x < y) { const uint32_t t = x; x = y; y = t; }
                        if (atomicCAS(&comp[x], x, y) == x) break;
                    }
                }
            }
        }
        __syncwarp();
        // one component (the usual case): its term folds every vertex and edge, so the per-root
        // sums -- shared-memory atomics that would all hit the one root -- are skipped
        uint32_t nroots = 0;
        for (uint32_t v = lane; v < V; v += 32) nroots += (deg[v] && comp[v] == v) ? 1u : 0u;
        one = warp_sum32(nroots) == 1;
    }
    uint64_t vs = 0, es = 0, cs = 0;
    for (uint32_t v = lane; v < V; v += 32) {
        if (!deg[v]) continue;
        const uint64_t m = smix(cur[v]);
        vs += m;
        if (one) continue;
        uint32_t r = v;
        while (comp[r] != r) r = comp[r];
        atomicAdd(reinterpret_cast<unsigned long long*>(&csum[r]), static_cast<unsigned long long>(m));
        atomicAdd(reinterpret_cast<unsigned long long*>(&ccnt[r]), 1ull);
    }
    for (uint32_t e = lane; e < ne; e += 32) {
        const uint32_t a = car[e], vo = cvo[e];
        uint64_t h = fnv(kFnvOffset, static_cast<uint64_t>(a));
        for (uint32_t q = 0; q < a; ++q) h = fnv(h, cur[vloc[vo + q]]);
        es += smix(h);
        if (a && !one) {
            uint32_t r = vloc[vo];
            while (comp[r] != r) r = comp[r];
            atomicAdd(reinterpret_cast<unsigned long long*>(&ccnt[r]), 1ull << 32);
        }
    }
    __syncwarp();
    if (!one)
        for (uint32_t v = lane; v < V; v += 32)
            if (deg[v] && comp[v] == v) cs += smix(fnv(fnv(kFnvOffset, ccnt[v]), csum[v]));
    vs = warp_sum64(vs);
    es = warp_sum64(es);
    cs = one ? smix(fnv(fnv(kFnvOffset, (static_cast<uint64_t>(ne) << 32) | nv), vs))
             : warp_sum64(cs);
    uint64_t h = kFnvOffset;
    h = fnv(h, nv);
    h = fnv(h, ne);
    h = fnv(h, vs);
    h = fnv(h, es);
    h = fnv(h, cs);
    __syncwarp();
    return h;
}



// ------------------------------------------------------------------------------------------
// Incremental match forwarding (reference: hypergraph/src/parallel_evolution.cpp:630-755,
// forward_existing_parent_matches; hypergraph/include/hypergraph/pattern_matcher.hpp:469-537,
// find_delta_matches). A state created by event c from parent p has as matches exactly
//   F = the parent's matches (= p's events, already in canonical order) avoiding c's consumed
//       edges, plus
//   D = matches using at least one edge c produced, found by joins seeded at each produced edge
//       in each LHS position and kept only when the seed position is the first position that
//       holds a produced edge (so each is found once);
// F and D are disjoint, and merging them by the canonical key (state positions in schedule
// order) gives the same sequence the full join enumerates. Edge ids are stable and positions are
// monotone in ids, so F stays sorted.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fwd_key(const DevRule& R, const uint16_t* pos) {
    uint64_t k = 0;
    for (uint32_t i = 0; i < R.n_lhs; ++i) k = (k << 16) | pos[R.sched[i]];
    return k;
}

// Delta matches of state `pa` into dkey2/dpos2, sorted by key. Returns their number, or kNone
// if more than kFwdCap (the state is then re-joined instead).
__device__ uint32_t fwd_collect_delta(const Layout& L, char* sm, const DevRule& R, const Parent& pa,
                                      uint32_t prod0) {
    const uint32_t lane = lane_id();
    const uint32_t n = R.n_lhs;
    uint8_t* sched2 = smp<uint8_t>(sm, L.o_sched2);
    uint64_t* dkey = smp<uint64_t>(sm, L.o_dkey);
    uint16_t* dpos = smp<uint16_t>(sm, L.o_dpos);
    uint64_t* dkey2 = smp<uint64_t>(sm, L.o_dkey2);
    uint16_t* dpos2 = smp<uint16_t>(sm, L.o_dpos2);
    const uint16_t* match = smp<uint16_t>(sm, L.o_match);
    uint32_t nd = 0;
    bool over = false;
    for (uint32_t x = prod0; x < pa.ne && !over; ++x) {
        for (uint32_t q = 0; q < n && !over; ++q) {
            if (lane == 0) {
                sched2[0] = static_cast<uint8_t>(q);
                uint32_t k = 1;
                for (uint32_t i = 0; i < n; ++i)
                    if (R.sched[i] != q) sched2[k++] = R.sched[i];
            }
            __syncwarp();
            warp_join(L, sm, R, pa, sched2, static_cast<int>(x), [&](uint32_t) {
                uint32_t first = n;
                for (uint32_t k = 0; k < n; ++k)
                    if (match[k] >= prod0) { first = k; break; }
                if (first != q || over) return;
                if (nd >= kFwdCap) { over = true; return; }
                if (lane < n) dpos[nd * kFwdMaxLhs + lane] = match[lane];
                if (lane == 0) dkey[nd] = fwd_key(R, match);
                ++nd;
                __syncwarp();
            });
        }
    }
    if (over) return kNone;
    __syncwarp();
    for (uint32_t i = lane; i < nd; i += 32) {
        const uint64_t k = dkey[i];
        uint32_t r = 0;
        for (uint32_t j = 0; j < nd; ++j) r += dkey[j] < k ? 1u : 0u;
        dkey2[r] = k;
        for (uint32_t t = 0; t < kFwdMaxLhs; ++t) dpos2[r * kFwdMaxLhs + t] = dpos[i * kFwdMaxLhs + t];
    }
    __syncwarp();
    return nd;
}

// State position of edge id `id` in the staged state (ids ascending).
__device__ __forceinline__ uint32_t fwd_find(const uint32_t* peid, uint32_t ne, uint32_t id) {
    uint32_t lo = 0, hi = ne;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (peid[mid] < id) lo = mid + 1; else hi = mid;
    }
    return lo;
}

struct Fwd {
    bool on;
    uint32_t e0, en;     // the parent's events
    uint32_t nk;         // consumed edges of the creating event (ids in smem o_fkc)
    uint32_t prod0;      // state position of the first produced edge
    uint32_t nd;         // delta matches (sorted in dkey2 / dpos2)
};

// Decide forwarding for a staged state and collect its delta matches.
__device__ Fwd fwd_prepare(const DevPtrs& P, const LevelArgs& A, const Layout& L, char* sm,
                           const DevRule& R, const DevEvo& ev, const Parent& pa, uint32_t sid,
                           bool want) {
    Fwd f;
    f.on = false;
    f.e0 = f.en = f.nk = f.prod0 = f.nd = 0;
    if (!want || A.fwd_mode == 0 || ev.rule_count != 1 || R.n_lhs > kFwdMaxLhs || R.n_rhs > pa.ne)
        return f;
    if (A.fwd_mode == 2 && pa.ne < 48) return f;
    const uint32_t c = P.st_event[sid];
    const uint32_t parent = c == kNone ? kNone : P.ev_in[c];
    if (parent == kNone) return f;   // a root
    uint32_t* kc = smp<uint32_t>(sm, L.o_fkc);
    const uint32_t lane = lane_id();
    const uint32_t co = P.ev_coff[c];
    if (lane < R.n_lhs) kc[lane] = P.ev_cons[co + lane];
    f.nk = R.n_lhs;
    f.e0 = P.st_ev0[parent];
    f.en = P.st_evn[parent];
    f.prod0 = pa.ne - R.n_rhs;
    __syncwarp();
    const uint32_t nd = fwd_collect_delta(L, sm, R, pa, f.prod0);
    if (nd == kNone) return f;
    f.nd = nd;
    f.on = true;
    return f;
}

// Forwarded parent matches, 32 at a time: for each one avoiding the consumed edges, its state
// positions (pattern order) and key into fkey/fpos[slot]. Returns how many of the 32 survived.
__device__ uint32_t fwd_chunk(const DevPtrs& P, const Layout& L, char* sm, const DevRule& R,
                              const Parent& pa, const Fwd& f, uint32_t base) {
    const uint32_t lane = lane_id();
    const uint32_t* kc = smp<uint32_t>(sm, L.o_fkc);
    const uint32_t* peid = smp<uint32_t>(sm, L.o_peid);
    uint64_t* fkey = smp<uint64_t>(sm, L.o_fkey);
    uint16_t* fpos = smp<uint16_t>(sm, L.o_fpos);
    bool valid = base + lane < f.en;
    uint16_t pos[kFwdMaxLhs] = {0, 0, 0, 0};
    if (valid) {
        const uint32_t e = f.e0 + base + lane;
        const uint32_t co = P.ev_coff[e];
        for (uint32_t k = 0; k < R.n_lhs && valid; ++k) {
            const uint32_t id = P.ev_cons[co + k];
            for (uint32_t m = 0; m < f.nk; ++m) valid &= kc[m] != id;
            pos[k] = static_cast<uint16_t>(fwd_find(peid, pa.ne, id));
        }
    }
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, valid);
    if (valid) {
        const uint32_t slot = __popc(bal & ((1u << lane) - 1u));
        fkey[slot] = fwd_key(R, pos);
        for (uint32_t k = 0; k < kFwdMaxLhs; ++k) fpos[slot * kFwdMaxLhs + k] = pos[k];
    }
    __syncwarp();
    return __popc(bal);
}

// Emit one match given by its state positions (pattern order): sets match / taken / binding
// exactly as the join does, then calls on_match.
template <class F>
__device__ void fwd_emit(const Layout& L, char* sm, const DevRule& R, const uint16_t* pos,
                         F&& on_match) {
    const uint32_t lane = lane_id();
    uint16_t* match = smp<uint16_t>(sm, L.o_match);
    uint32_t* taken = smp<uint32_t>(sm, L.o_taken);
    uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint32_t nm = 0;
    for (uint32_t k = 0; k < R.n_lhs; ++k) {
        const uint32_t e = pos[k];
        const uint32_t a = R.lhs_ar[k], vo = pevo[e];
        for (uint32_t q = 0; q < a; ++q) {
            const uint32_t var = R.lhs_vars[R.lhs_off[k] + q];
            if (lane == 0) bind[var] = vloc[vo + q];
            nm |= 1u << var;
        }
        if (lane == 0) {
            match[k] = static_cast<uint16_t>(e);
            taken[e >> 5] |= 1u << (e & 31u);
        }
    }
    __syncwarp();
    on_match(nm);
    __syncwarp();
    if (lane == 0)
        for (uint32_t k = 0; k < R.n_lhs; ++k) taken[pos[k] >> 5] &= ~(1u << (pos[k] & 31u));
    __syncwarp();
}

// Every match of the staged state in canonical order: the full join, or forwarding.
template <class F, class Skip = NoSkip>
__device__ void enumerate_matches(const DevPtrs& P, const Layout& L, char* sm, const DevRule& R,
                                  const Parent& pa, const Fwd& f, F&& on_match,
                                  uint32_t limit = 0xFFFFFFFFu, Skip skip = Skip()) {
    if (!f.on) {
        warp_join(L, sm, R, pa, R.sched, -1, on_match, limit, skip);
        return;
    }
    const uint32_t lane = lane_id();
    uint32_t* taken = smp<uint32_t>(sm, L.o_taken);
    for (uint32_t w = lane; w < L.W; w += 32) taken[w] = 0;
    __syncwarp();
    const uint64_t* dkey2 = smp<uint64_t>(sm, L.o_dkey2);
    const uint16_t* dpos2 = smp<uint16_t>(sm, L.o_dpos2);
    const uint64_t* fkey = smp<uint64_t>(sm, L.o_fkey);
    const uint16_t* fpos = smp<uint16_t>(sm, L.o_fpos);
    uint32_t j = 0;
    for (uint32_t base = 0; base < f.en; base += 32) {
        const uint32_t m = fwd_chunk(P, L, sm, R, pa, f, base);
        for (uint32_t t = 0; t < m; ++t) {
            while (j < f.nd && dkey2[j] < fkey[t]) fwd_emit(L, sm, R, dpos2 + j++ * kFwdMaxLhs, on_match);
            fwd_emit(L, sm, R, fpos + t * kFwdMaxLhs, on_match);
        }
        __syncwarp();
    }
    while (j < f.nd) fwd_emit(L, sm, R, dpos2 + j++ * kFwdMaxLhs, on_match);
}

// Number of matches under forwarding (F survivors + D).
__device__ uint32_t fwd_count(const DevPtrs& P, const Layout& L, char* sm, const DevRule& R,
                              const Parent& pa, const Fwd& f) {
    uint32_t c = f.nd;
    for (uint32_t base = 0; base < f.en; base += 32) c += fwd_chunk(P, L, sm, R, pa, f, base);
    return c;
}

// ------------------------------------------------------------------------------------------
// Lane-per-child WL. For the small states that dominate deep evolutions (a handful of
// vertices, tens of edges) one warp per child leaves most lanes idle; instead the warp stages
// the parent once, enumerates up to 32 matches into a batch, and every lane hashes one child
// against the shared parent. A child is described by the parent positions it removes and the
// local vertex ids of its produced edges; its occurrence lists are the parent's (edge order)
// minus removed edges, followed by the produced occurrences (RHS order) -- the child's edge
// order, so the initial-colour truncation sees occurrences in the same order as the reference.
// ------------------------------------------------------------------------------------------
__device__ uint32_t build_parent_csr(const Layout& L, char* sm, const Parent& pa) {
    const uint32_t lane = lane_id();
    const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
    const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
    const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
    uint16_t* poff = smp<uint16_t>(sm, L.o_poff);
    uint16_t* pocc = smp<uint16_t>(sm, L.o_pocc);
    uint16_t* pdeg = smp<uint16_t>(sm, L.o_pdeg);
    uint16_t* pnn = smp<uint16_t>(sm, L.o_pnn);
    uint16_t* pnoff = smp<uint16_t>(sm, L.o_pnoff);
    uint16_t* pnbr = smp<uint16_t>(sm, L.o_pnbr);
    uint32_t* pcnt = smp<uint32_t>(sm, L.o_pcnt);
    const uint32_t v = lane;
    uint32_t d = 0, nn = 0, adj = 0;   // adj: vertices sharing an edge with v (nvp <= 32)
    uint32_t cnt = 0;                  // occurrences of v by position (byte q, positions < 4)
    const uint32_t a0 = pa.ne ? pear[0] : 0u;
    bool uni = a0 >= 2 && a0 <= 4;     // every edge has arity a0 (lanes check their share)
    for (uint32_t e = lane; e < pa.ne; e += 32) uni = uni && pear[e] == a0;
    uni = __all_sync(0xFFFFFFFFu, uni);
    if (v < pa.nvp)
        for (uint32_t e = 0; e < pa.ne; ++e) {
            const uint32_t a = pear[e], vo = pevo[e];
            for (uint32_t q = 0; q < a; ++q)
                if (vloc[vo + q] == v) {
                    ++d;
                    nn += a - 1;
                    cnt += q < 4 ? 1u << (8 * q) : 0u;
                    for (uint32_t k = 0; k < a; ++k) adj |= 1u << vloc[vo + k];
                }
        }
    // connectivity: grow the set reached from vertex 0 (at most nvp rounds)
    uint32_t reach = pa.nvp ? 1u : 0u;
    for (uint32_t it = 0; it < pa.nvp; ++it) {
        const uint32_t nr = reach | __reduce_or_sync(0xFFFFFFFFu, ((reach >> lane) & 1u) ? adj : 0u);
        if (nr == reach) break;
        reach = nr;
    }
    const uint32_t inc = warp_incl_scan(d);
    const uint32_t incn = warp_incl_scan(nn);
    if (v < pa.nvp) {
        pcnt[v] = cnt;
        poff[v] = static_cast<uint16_t>(inc - d);
        pdeg[v] = static_cast<uint16_t>(d);
        pnn[v] = static_cast<uint16_t>(nn);
        pnoff[v] = static_cast<uint16_t>(incn - nn);
        uint32_t w = inc - d, wn = incn - nn;
        for (uint32_t e = 0; e < pa.ne; ++e) {
            const uint32_t a = pear[e], vo = pevo[e];
            for (uint32_t q = 0; q < a; ++q) {
                if (vloc[vo + q] != v) continue;
                pocc[w++] = static_cast<uint16_t>((e << 4) | q);
                for (uint32_t k = 0; k < a; ++k)
                    if (k != q) pnbr[wn++] = lane_nbr_entry(e, vloc[vo + k], k);
            }
        }
    }
    if (lane == 31) {
        poff[pa.nvp] = static_cast<uint16_t>(inc);
        pnoff[pa.nvp] = static_cast<uint16_t>(incn);
        const uint32_t all = pa.nvp >= 32 ? 0xFFFFFFFFu : (1u << pa.nvp) - 1u;
        *smp<uint32_t>(sm, L.o_pconn) = ((pa.nvp && reach == all) ? 1u : 0u) | ((uni ? a0 : 0u) << 8);
    }
    const uint32_t nnmax = warp_max32(nn);
    __syncwarp();
    return nnmax;
}

template <int VM, int NM>
__device__ __forceinline__ uint64_t lane_wl(const Layout& L, char* sm, const Parent& pa,
                                            const DevRule& R, const uint8_t* slot, WlInfo& info) {
    return lane_wl_core<VM, NM>(smp<uint8_t>(sm, L.o_pear), smp<uint16_t>(sm, L.o_pevo),
                                smp<uint16_t>(sm, L.o_vloc), smp<uint16_t>(sm, L.o_poff),
                                smp<uint16_t>(sm, L.o_pocc), smp<uint16_t>(sm, L.o_pdeg),
                                smp<uint16_t>(sm, L.o_pnn), smp<uint16_t>(sm, L.o_pnoff),
                                smp<uint16_t>(sm, L.o_pnbr), smp<uint32_t>(sm, L.o_pcnt),
                                *smp<uint32_t>(sm, L.o_pconn), pa.ne, pa.nvp, R, slot, info);
}

}  // namespace

// ==========================================================================================
// Kernels
// ==========================================================================================

// Root states: hash the uploaded records and seed the dedup tables.
__global__ void k_roots(DevPtrs P, const uint32_t* sids, uint32_t n, uint32_t* work, Layout L) {
    extern __shared__ __align__(16) char smem[];
    char* sm = smem + (threadIdx.x >> 5) * L.bytes;
    const uint32_t lane = lane_id();
    WarpWork q;
    while (true) {
        const uint32_t i = q.next(work);
        if (i >= n) break;
        const uint32_t sid = sids[i];
        const Parent pa = load_parent(P, L, sm, sid);
        uint8_t* car = smp<uint8_t>(sm, L.o_car);
        uint16_t* cvo = smp<uint16_t>(sm, L.o_cvo);
        const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
        const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
        for (uint32_t e = lane; e < pa.ne; e += 32) { car[e] = pear[e]; cvo[e] = pevo[e]; }
        __syncwarp();
        WlInfo info;
        const uint64_t h = warp_wl(L, sm, pa.ne, pa.nvp, info);
        if (lane == 0) {
            P.st_hash[sid] = h;
            P.st_nv[sid] = pa.nvp;
            const uint32_t a = P.st_event[sid];
            P.ev_hash[a] = h;
            table_insert(P, P.evos[P.st_evo[sid]], h, a);
        }
        __syncwarp();
    }
}

// Count the matches of every (frontier state, rule) item. Held to 64 registers (4 blocks per
// SM; no spills): its latency-bound walk needs the warps (C2 count 1.00 -> 0.65 ms).
__global__ void __launch_bounds__(256, 4) k_count(DevPtrs P, LevelArgs A, Layout L) {
    extern __shared__ __align__(16) char smem[];
    char* sm = smem + (threadIdx.x >> 5) * L.bytes;
    const uint32_t lane = lane_id();
    const DevRule& R = *smp<DevRule>(sm, L.o_rule);
    uint32_t max_cnt = 0;   // largest match count of a (state, rule) this warp counted
    WarpWork q;
    while (true) {
        const uint32_t f = q.next(&A.work[0]);
        if (f >= A.n_frontier) break;
        const uint32_t sid = A.frontier[f];
        const Parent pa = load_parent(P, L, sm, sid);
        build_join_index(L, sm, pa);
        const DevEvo ev = P.evos[P.st_evo[sid]];
        // lane-per-child eligibility: few enough vertices and a bounded neighbour count
        bool lane_ok = pa.nvp <= A.lane_vmax && pa.ne <= kLaneEMax && pa.ne > 0;
        uint32_t pnn_max = 0;
        if (lane_ok) {
            const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
            const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
            const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
            uint32_t nn = 0;
            if (lane < pa.nvp)
                for (uint32_t e = 0; e < pa.ne; ++e)
                    for (uint32_t q = 0; q < pear[e]; ++q)
                        if (vloc[pevo[e] + q] == lane) nn += pear[e] - 1u;
            pnn_max = warp_max32(nn);
        }
        bool fwd_on = false;
        for (uint32_t r = 0; r < A.rules_stride; ++r) {
            uint32_t cnt = 0;
            if (r < ev.rule_count) {
                load_rule(sm, L, &P.rules[ev.rule_begin + r]);
                uint32_t gain = 0;
                for (uint32_t k = 0; k < R.n_rhs; ++k) gain += uint32_t(R.rhs_ar[k]) * (R.rhs_ar[k] - 1u);
                lane_ok = lane_ok && pa.nvp + R.n_fresh <= A.lane_vmax && pnn_max + gain <= kLaneNMax;
                const Fwd fw = fwd_prepare(P, A, L, sm, R, ev, pa, sid, true);
                fwd_on = fw.on;
                if (fw.on) cnt = fwd_count(P, L, sm, R, pa, fw);
                else if (pa.ne <= kLaneEMax && R.n_lhs <= kLaneJoinLhs) cnt = lane_join_count(L, sm, R, pa);
                else warp_join(L, sm, R, pa, R.sched, -1, [&](uint32_t) { ++cnt; }, 0xFFFFFFFFu,
                               SkipCounter{&cnt, 0xFFFFFFFFu});
            }
            if (lane == 0) A.counts[f * A.rules_stride + r] = cnt;
            max_cnt = max(max_cnt, cnt);
            __syncwarp();
        }
        if (lane == 0) A.fmode[f] = (lane_ok ? 1 : 0) | (fwd_on ? 2 : 0);
    }
    if (lane == 0 && max_cnt) atomicMax(&A.level_max[4], max_cnt);   // sizes the staged match list
}

// Per-item counts scaled by the rule's consumed / produced / fresh sizes, for the scans.
__global__ void k_item_sizes(DevPtrs P, LevelArgs A) {
    const uint32_t n = A.n_frontier * A.rules_stride;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t f = t / A.rules_stride, r = t % A.rules_stride;
        const uint32_t sid = A.frontier[f];
        const DevEvo& ev = P.evos[P.st_evo[sid]];
        const uint32_t c = A.counts[t];
        uint32_t cons = 0, prod = 0, fresh = 0;
        if (r < ev.rule_count && c) {
            const DevRule& R = P.rules[ev.rule_begin + r];
            cons = c * R.n_lhs;
            prod = c * R.n_rhs;
            fresh = c * R.n_fresh;
        }
        A.item_ev[t] = c;
        A.item_cons[t] = cons;
        A.item_prod[t] = prod;
        A.item_fresh[t] = fresh;
    }
}

// An event's consumed parent positions as a bit mask for the branchial test (events of one input
// state share the parent's positions, so equal positions are equal edges), or 0 when the parent
// has more than 63 edges (the test then compares edge ids). Bit 63 is never a position: an event
// that is not kept carries kMaskDropped, which shares no position with any other mask.
constexpr unsigned long long kMaskDropped = 1ull << 63;

__device__ __forceinline__ unsigned long long branch_mask(uint32_t n, uint32_t pne, const uint8_t* pos) {
    if (pne > 63) return 0ull;
    unsigned long long m = 0;
    for (uint32_t k = 0; k < n; ++k) m |= 1ull << pos[k];
    return m;
}

// Frontier position of work index w (identity unless the level runs over a list of ranges).
__device__ __forceinline__ uint32_t frontier_at(const LevelArgs& A, uint32_t w) {
    if (!A.frng) return w;
    const uint32_t* off = A.frng + A.n_frng;
    uint32_t a = 0, b = A.n_frng;   // off[a] <= w < off[b]
    while (b - a > 1) {
        const uint32_t m = (a + b) >> 1;
        if (off[m] <= w) a = m; else b = m;
    }
    return A.frng[a] + (w - off[a]);
}

// Children per slice of a parent hashed warp-per-child: the smallest power of two >= 4 and
// >= sqrt(children), so a parent with many children is spread over about sqrt(children) warps
// while each warp re-enumerates at most its slice's end of the parent's matches.
__device__ __forceinline__ uint32_t slice_size(uint32_t children) {
    uint32_t s = 4;
    while (uint64_t(s) * s < children) s <<= 1;
    return s;
}

__device__ __forceinline__ uint32_t children_of(const LevelArgs& A, uint32_t f) {
    return A.item_ev[(f + 1) * A.rules_stride] - A.item_ev[f * A.rules_stride];
}

// Slice counts of the work indices [f_begin, f_begin + n) for the warp-per-child kernel.
__global__ void k_slice_counts(LevelArgs A, uint32_t n, uint32_t* cnt) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
        const uint32_t f = frontier_at(A, A.f_begin + w);
        const uint32_t c = children_of(A, f);
        cnt[w] = ((A.fmode[f] & 1u) || !c) ? 0u : (c + slice_size(c) - 1) / slice_size(c);
    }
}

// Enumerate again; mint events, produced edges and fresh vertices at the scanned offsets;
// hash every child; insert the hash into the dedup table. Two instantiations over the same
// frontier range: kLane hashes the children of the states flagged by k_count one per lane,
// the other one child per warp (states too large for a lane's private arrays).
// kWalk (lane kernel only): matches of small states come from the lane-parallel join, staged in
// shared memory; without it the warp join enumerates them into the batch directly. The two are
// separate instantiations because the walk's code costs the other path registers and issue slots.
template <bool kLane, bool kWalk = false>
__global__ void __launch_bounds__(256, 3) k_expand(DevPtrs P, LevelArgs A, Layout L) {
    extern __shared__ __align__(16) char smem[];
    char* sm = smem + (threadIdx.x >> 5) * L.bytes;
    const uint32_t lane = lane_id();
    const DevRule& R = *smp<DevRule>(sm, L.o_rule);
    const uint32_t* peid = smp<uint32_t>(sm, L.o_peid);
    const uint16_t* match = smp<uint16_t>(sm, L.o_match);
    const uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
    uint8_t* batch = smp<uint8_t>(sm, L.o_batch);
    uint64_t b_stage = 0, b_hbm = 0, n_child = 0, n_rounds = 0;   // per-lane accumulators
    uint32_t* work = &A.work[kLane ? 1 : 2];
    WarpWork q;
    while (true) {
        const uint32_t u = q.next(work);
        // the parent's children [c_lo, c_hi) (in its child order over all rules) built by this unit
        uint32_t f, c_lo = 0, c_hi = 0xFFFFFFFFu;
        if (kLane || !A.soff) {
            if (u >= A.f_end - A.f_begin) break;
            f = frontier_at(A, A.f_begin + u);
        } else {
            if (u >= A.soff[A.n_sw]) break;
            uint32_t a = 0, b = A.n_sw;   // the work index whose slices hold u
            while (b - a > 1) {
                const uint32_t m = (a + b) >> 1;
                if (A.soff[m] <= u) a = m; else b = m;
            }
            f = frontier_at(A, A.f_begin + a);
            const uint32_t S = slice_size(children_of(A, f));
            c_lo = (u - A.soff[a]) * S;
            c_hi = c_lo + S;
        }
        const uint8_t fm = A.fmode[f];
        if (((fm & 1u) != 0) != kLane) continue;
        const uint32_t sid = A.frontier[f];
        const Parent pa = load_parent(P, L, sm, sid);
        const uint32_t evo = P.st_evo[sid];
        const DevEvo ev = P.evos[evo];
        if (lane == 0 && c_lo == 0) b_hbm += 4ull * (pa.ne + (pa.ne + 3) / 4 + pa.nocc) + 20;
        if (kLane) build_parent_csr(L, sm, pa);
        else build_join_index(L, sm, pa);
        // warp path: whether the parent is one component (then so is every child of a rule whose
        // right-hand side joins its left-hand vertices, and warp_wl skips its union-find)
        const bool pconn = !kLane && parent_connected(L, sm, pa);
        for (uint32_t r = 0; r < A.rules_stride && r < ev.rule_count; ++r) {
            const uint32_t item = f * A.rules_stride + r;
            if (lane == 0 && c_lo == 0) b_stage += 4ull * pa.ne + 4ull * pa.nocc;   // join: ids and vertices
            const uint32_t rn = A.counts[item];
            const uint32_t rb = A.item_ev[item] - A.item_ev[f * A.rules_stride];
            if (rn == 0 || rb + rn <= c_lo || rb >= c_hi) continue;
            load_rule(sm, L, &P.rules[ev.rule_begin + r]);
            const uint32_t ev0 = A.ev_base + A.item_ev[item];
            const uint32_t cons0 = A.cons_base + A.item_cons[item];
            const uint32_t prod0 = A.prod_base + A.item_prod[item];
            const uint32_t fresh0 = A.fresh_base + A.item_fresh[item];
            const uint32_t rule_g = ev.rule_begin + r;
            const Fwd fwd = fwd_prepare(P, A, L, sm, R, ev, pa, sid, (fm & 2u) != 0);
            // per-child work shared by both paths: the event record and the table insert
            auto finish = [&](uint32_t idx, uint64_t h, const WlInfo& info, const uint8_t* rpos) {
                const uint32_t e = ev0 + idx;
                const uint32_t coff = cons0 + idx * R.n_lhs;
                const uint32_t pid = prod0 + idx * R.n_rhs;
                P.ev_in[e] = sid;
                P.ev_rule[e] = rule_g;
                P.ev_coff[e] = coff;
                P.ev_prod[e] = pid;
                P.ev_fresh[e] = fresh0 + idx * R.n_fresh;
                P.ev_hash[e] = h;
                P.ev_nv[e] = info.nv;
                for (uint32_t k = 0; k < R.n_lhs; ++k) P.ev_cons[coff + k] = peid[rpos[k]];
                P.ev_bmask[e] = branch_mask(R.n_lhs, pa.ne, rpos);
                for (uint32_t k = 0; k < R.n_rhs; ++k) P.edge_creator[pid + k] = e;
                table_insert(P, ev, h, e);
                const uint64_t k = R.n_lhs, rr = R.n_rhs;
                const uint32_t nec = pa.ne - R.n_lhs + R.n_rhs;
                b_stage += 4 * k + 8;
                b_stage += 4ull * pa.ne + 4ull * nec + 4ull * R.rhs_total + 12 * rr + 16 + 4 * k + 4 * rr;
                b_stage += 5ull * info.nocc + 8ull * info.nv +
                           uint64_t(info.rounds) * (8ull * info.nbr + 5ull * info.nocc + 16ull * info.nv) +
                           8ull * info.nv + 8ull * info.nocc;
                b_stage += 16;
                b_hbm += 20 + 8 + 8 * k + 4 * rr + 16;
                n_child += 1;
                n_rounds += info.rounds;
            };
            if constexpr (kLane) {
              if (kWalk && !fwd.on && pa.ne <= kLaneEMax && R.n_lhs <= kLaneJoinLhs && rn <= L.MCAP) {
                // stage the rule's matches in canonical order (lane walks: count, scan, emit),
                // then hash them 32 at a time, one child per lane
                uint32_t* mlist = smp<uint32_t>(sm, L.o_mlist);
                const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
                const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
                uint32_t total = 0;
                for (uint32_t b = 0; b < pa.ne; b += 32) {
                    const uint32_t e0 = b + lane;
                    const uint32_t c = e0 < pa.ne ? lane_walk(L, sm, R, pa, e0, [](uint32_t) {}) : 0u;
                    const uint32_t inc = warp_incl_scan(c);
                    uint32_t w = total + inc - c;
                    if (c) lane_walk(L, sm, R, pa, e0, [&](uint32_t pk) {
                        if (w < L.MCAP) mlist[w] = pk;
                        ++w;
                    });
                    total += __shfl_sync(0xFFFFFFFFu, inc, 31);
                }
                __syncwarp();
                if (total != rn) {
                    if (lane == 0) atomicOr(P.err, kErrJoinCount);
                    continue;
                }
                for (uint32_t b = 0; b < rn; b += 32) {
                    const uint32_t i = b + lane;
                    if (i < rn) {
                        uint8_t* slot = batch + lane * L.SB;
                        const uint32_t pk = mlist[i];
                        uint16_t bv[kMaxVars];
                        for (uint32_t k = 0; k < R.n_lhs; ++k) {
                            const uint32_t pos = (pk >> (8u * k)) & 0xFFu;
                            slot[k] = static_cast<uint8_t>(pos);
                            const uint32_t vo = pevo[pos];
                            for (uint32_t q = 0; q < R.lhs_ar[k]; ++q)
                                bv[R.lhs_vars[R.lhs_off[k] + q]] = vloc[vo + q];
                        }
                        for (uint32_t t = 0; t < R.rhs_total; ++t) {
                            const uint32_t var = R.rhs_vars[t];
                            slot[R.n_lhs + t] = static_cast<uint8_t>(((R.new_mask >> var) & 1u)
                                                                     ? pa.nvp + R.fresh_rank[var]
                                                                     : bv[var]);
                        }
                        WlInfo info;
                        const uint64_t h = lane_wl<kLaneVMax, kLaneNMax>(L, sm, pa, R, slot, info);
                        finish(i, h, info, slot);
                    }
                    __syncwarp();
                }
              } else {
                uint32_t nb = 0, done = 0;
                auto flush = [&]() {
                    if (lane < nb) {
                        const uint8_t* slot = batch + lane * L.SB;
                        WlInfo info;
                        const uint64_t h = lane_wl<kLaneVMax, kLaneNMax>(L, sm, pa, R, slot, info);
                        finish(done + lane, h, info, slot);
                    }
                    __syncwarp();
                    done += nb;
                    nb = 0;
                };
                enumerate_matches(P, L, sm, R, pa, fwd, [&](uint32_t nm) {
                    uint8_t* slot = batch + nb * L.SB;
                    if (lane < R.n_lhs) slot[lane] = static_cast<uint8_t>(match[lane]);
                    for (uint32_t t = lane; t < R.rhs_total; t += 32) {
                        const uint32_t var = R.rhs_vars[t];
                        slot[R.n_lhs + t] = static_cast<uint8_t>(((nm >> var) & 1u) ? bind[var]
                                                                 : pa.nvp + R.fresh_rank[var]);
                    }
                    __syncwarp();
                    if (++nb == 32) flush();
                });
                if (nb) flush();
              }
            } else {
                // this rule's children inside the unit's slice: [lo, hi) of its match order
                const uint32_t lo = c_lo > rb ? c_lo - rb : 0u;
                const uint32_t hi = min(rn, c_hi - rb);
                uint32_t idx = 0;
                uint8_t rpos[kMaxPatternEdges];
                // matches before the slice are skipped whole at the last position (popcounts)
                enumerate_matches(P, L, sm, R, pa, fwd, [&](uint32_t nm) {
                    if (idx >= lo && idx < hi) {
                        for (uint32_t k = 0; k < R.n_lhs; ++k) rpos[k] = static_cast<uint8_t>(match[k]);
                        const uint32_t nec = build_child(L, sm, R, pa, nm);
                        WlInfo info;
                        const uint64_t h = warp_wl(L, sm, nec, pa.nvp + R.n_fresh, info,
                                                   pconn && (R.flags & kRuleRhsJoinsLhs));
                        if (lane == 0) finish(idx, h, info, rpos);
                        __syncwarp();
                    }
                    ++idx;
                }, hi, SkipCounter{&idx, lo});
            }
        }
    }
    b_stage = warp_sum64(b_stage);
    b_hbm = warp_sum64(b_hbm);
    n_child = warp_sum64(n_child);
    n_rounds = warp_sum64(n_rounds);
    if (lane == 0 && b_hbm) {
        unsigned long long* st = P.stats + (kLane ? 0 : 4);
        atomicAdd(&st[0], static_cast<unsigned long long>(b_stage));
        atomicAdd(&st[1], static_cast<unsigned long long>(b_hbm));
        atomicAdd(&st[2], static_cast<unsigned long long>(n_child));
        atomicAdd(&st[3], static_cast<unsigned long long>(n_rounds));
    }
}

// Producer event of every consumed edge of the level's built events (the causal relation's
// gather: an edge has exactly one producer, recorded when it was minted).
__global__ void k_cprod(DevPtrs P, uint32_t ev_base, uint32_t n) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t e = ev_base + t;
        const uint32_t co = P.ev_coff[e], k = P.rules[P.ev_rule[e]].n_lhs;
        for (uint32_t i = 0; i < k; ++i) P.ev_cprod[co + i] = P.edge_creator[P.ev_cons[co + i]];
    }
}

// Transitive reduction of the causal relation, one level at a time (after k_cprod).
//
// Every producer of an edge consumed by event c created an edge of c's input state, so it lies on
// that state's history chain (root -> ... -> input state, one creating event per level), and so
// do all of its own causal ancestors. An event's causal ancestors are therefore identified by
// their levels: anc(c) = OR over c's producers q of (bit level(q) | anc(q)). A pair (p, c) is
// implied by a longer path exactly when another producer q of c has p among its ancestors
// (bit level(p) in anc(q)); such consumed positions get producer kNone, which removes their
// triples from every causal output. Reachability over the reduced pairs equals reachability over
// all pairs, so anc stays exact for later levels. The result is the unique transitive reduction
// of the stored (producer, consumer) relation that the reference computes
// (common/include/hgcommon/transitive_reduction.hpp:36-94; kept triples: those whose pair
// survives, hypergraph/include/hypergraph/causal_graph.hpp:295-305).
__global__ void k_tr(DevPtrs P, uint32_t ev_base, uint32_t n) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t e = ev_base + t;
        const uint32_t co = P.ev_coff[e], k = P.rules[P.ev_rule[e]].n_lhs;
        uint32_t q[kMaxPatternEdges];
        uint32_t lv[kMaxPatternEdges];
        unsigned long long qa[kMaxPatternEdges];
        unsigned long long anc = 0;
        bool deep = false;
        for (uint32_t i = 0; i < k; ++i) {
            q[i] = P.ev_cprod[co + i];
            lv[i] = 0;
            qa[i] = 0;
            if (q[i] == kNone) continue;
            lv[i] = P.st_depth[P.ev_in[q[i]]];
            deep |= lv[i] >= 64;
            qa[i] = P.ev_anc[q[i]];
            anc |= qa[i] | (1ull << (lv[i] & 63u));
        }
        P.ev_anc[e] = anc;
        if (deep) { atomicOr(P.err, kErrTrDepth); continue; }
        for (uint32_t i = 0; i < k; ++i) {
            if (q[i] == kNone) continue;
            bool implied = false;
            for (uint32_t j = 0; j < k && !implied; ++j)
                implied = q[j] != kNone && q[j] != q[i] && ((qa[j] >> lv[i]) & 1ull);
            if (implied) P.ev_cprod[co + i] = kNone;
        }
    }
}




// Per frontier state: its first event and first-rule event count (the record match forwarding
// reads at the next level). Per evolution: first / one-past-last event of this level (the
// frontier is grouped by evolution, so each evolution's items are contiguous), and its cap cut
// reset. For the level: the frontier's largest edge and occurrence counts (level_max[2..3], they
// size the expand layouts) and how many states with children are off the lane path
// (level_max[5]; none: the warp-path launches are skipped).
__global__ void k_frontier_events(DevPtrs P, LevelArgs A, uint32_t* evo_last, uint32_t* evo_frange) {
    uint32_t mne = 0, mno = 0, mnv = 0, n_warp = 0;
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < A.n_frontier;
         f += gridDim.x * blockDim.x) {
        const uint32_t sid = A.frontier[f];
        const uint32_t t = f * A.rules_stride;
        P.st_ev0[sid] = A.ev_base + A.item_ev[t];
        P.st_evn[sid] = A.item_ev[t + 1] - A.item_ev[t];
        mne = max(mne, P.st_ne[sid]);
        mno = max(mno, P.st_nocc[sid]);
        mnv = max(mnv, P.st_nv[sid]);
        const bool children = A.item_ev[t + A.rules_stride] != A.item_ev[t];
        n_warp += (!(A.fmode[f] & 1u) && children) ? 1u : 0u;
        const uint32_t evo = P.st_evo[sid];
        if (f == 0 || P.st_evo[A.frontier[f - 1]] != evo) {
            P.evo_first_ev[evo] = A.ev_base + A.item_ev[f * A.rules_stride];
            P.evo_cut[evo] = kNone;
            evo_frange[2 * evo] = f;
        }
        if (f + 1 == A.n_frontier || P.st_evo[A.frontier[f + 1]] != evo) {
            evo_last[evo] = A.ev_base + A.item_ev[(f + 1) * A.rules_stride];
            evo_frange[2 * evo + 1] = f + 1;
        }
    }
    mne = warp_max32(mne);
    mno = warp_max32(mno);
    mnv = warp_max32(mnv);
    n_warp = warp_sum32(n_warp);
    if (lane_id() == 0) {
        atomicMax(&A.level_max[2], mne);
        atomicMax(&A.level_max[3], mno);
        atomicMax(&A.level_max[6], mnv);
        if (n_warp) atomicAdd(&A.level_max[5], n_warp);
    }
}

// Per evolution of the level: its kept events, its new states and its branchial pairs are each
// one contiguous range (the frontier is grouped by evolution and everything is numbered in
// frontier order). out[evo * 7 + {0..6}] = event first/end, state first/end, pair first/end, and
// the evolution's states in the next frontier.
// A level's first read-back in one copy: out[0..2] = event / consumed, produced / fresh totals and
// the frontier's largest edge / occurrence counts (low | high << 32), out[3] the largest match
// count of a (state, rule) | frontier states for the warp path << 32, then per evolution its
// classes, states, event signatures (sigs may be null) and first | last event << 32.
__global__ void k_sync1_pack(const uint32_t* item_ev, const uint32_t* item_cons,
                             const uint32_t* item_prod, const uint32_t* item_fresh, uint32_t ni,
                             const uint32_t* level_max, const unsigned long long* classes,
                             const unsigned long long* states, const unsigned long long* sigs,
                             const uint32_t* first, const uint32_t* last, uint32_t nevo,
                             unsigned long long* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    using u64 = unsigned long long;
    if (t == 0) {
        out[0] = item_ev[ni] | (u64(item_cons[ni]) << 32);
        out[1] = item_prod[ni] | (u64(item_fresh[ni]) << 32);
        out[2] = level_max[2] | (u64(level_max[3]) << 32);
        out[3] = level_max[4] | (u64(level_max[5]) << 32);
        out[4] = level_max[6];
    }
    for (uint32_t e = t; e < nevo; e += gridDim.x * blockDim.x) {
        out[5 + e] = classes[e];
        out[5 + nevo + e] = states[e];
        out[5 + 2ull * nevo + e] = sigs ? sigs[e] : 0ull;
        out[5 + 3ull * nevo + e] = first[e] | (u64(last[e]) << 32);
    }
}

// The level's second read-back rides behind the per-evolution ranges: new states, next-frontier
// states, branchial pairs and the error flags.
// out[4..8]: evolution 0's class and state counters and its stopped flag (final for the range:
// k_rep has run), which the level's range loop and the next level's prefix estimate read without
// round trips of their own.
__global__ void k_sync2_pack(const uint32_t* flag_rep, const uint32_t* flag_front,
                             const uint32_t* boff, uint32_t ne2, const uint32_t* err,
                             const unsigned long long* classes, const unsigned long long* states,
                             const uint32_t* stopped, uint32_t* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[0] = flag_rep[ne2];
        out[1] = flag_front[ne2];
        out[2] = boff[ne2];
        out[3] = *err;
        out[4] = static_cast<uint32_t>(classes[0]);
        out[5] = static_cast<uint32_t>(classes[0] >> 32);
        out[6] = static_cast<uint32_t>(states[0]);
        out[7] = static_cast<uint32_t>(states[0] >> 32);
        out[8] = stopped[0];
    }
}

__global__ void k_evo_ranges(DevPtrs P, LevelArgs A, const uint32_t* evo_last, uint32_t* out) {
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < A.n_frontier;
         f += gridDim.x * blockDim.x) {
        const uint32_t evo = P.st_evo[A.frontier[f]];
        if (f != 0 && P.st_evo[A.frontier[f - 1]] == evo) continue;
        const uint32_t e0 = P.evo_first_ev[evo];
        uint32_t e1 = min(evo_last[evo], A.ev_base + A.n_events);
        e1 = max(e0, min(e1, P.evo_cut[evo]));
        uint32_t* o = out + 7ull * evo;
        o[0] = e0;
        o[1] = e1;
        o[2] = A.state_base + A.flag_rep[e0 - A.ev_base];
        o[3] = A.state_base + A.flag_rep[e1 - A.ev_base];
        o[4] = A.bbase + A.boff[e0 - A.ev_base];
        o[5] = A.bbase + A.boff[e1 - A.ev_base];
        o[6] = A.flag_front[e1 - A.ev_base] - A.flag_front[e0 - A.ev_base];
    }
}

// ------------------------------------------------------------------------------------------
// Lane-per-child expansion with batches that cross parents (single-rule evolutions). A warp keeps
// kReg parent regions in shared memory (used in turn) and one 32-child batch: the children of the
// parent staged in one region are appended while other regions' leftover children are still
// waiting, so a parent with 38 children and the next one fill two batches instead of three. A
// region is restaged only once the batch holds none of its children. Children keep their own event ids,
// so the order in which batches are hashed changes nothing in the result.
// ------------------------------------------------------------------------------------------
struct LaneRegion {
    uint32_t sid, ev0, cons0, prod0, fresh0, rule_g, ne, nocc, nvp;
    uint64_t table_off, table_mask;
};

// kFwd = false: a level without match forwarding, compiled without its paths (a smaller kernel).
// The walk instantiation is held to 4 blocks per SM (64 registers; measured faster on small-state
// levels), the warp-join one to 3.
template <bool kWalk, int kReg = 2, bool kFwd = true>
__global__ void __launch_bounds__(256, kWalk ? 4 : 3) k_expand_lanes2(DevPtrs P, LevelArgs A, Layout L) {
    extern __shared__ __align__(16) char smem[];
    __shared__ LaneRegion rinfo_sm[8][kReg];
    __shared__ uint32_t meta_sm[8][32];
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t lane = lane_id();
    // region 0 carries the warp's batch and match list at its end; regions >= 1 stop before them
    char* const wbase = smem + w * (L.bytes + (kReg - 1) * L.region_bytes);
    auto rg = [&](uint32_t r) { return r == 0 ? wbase : wbase + L.bytes + (r - 1) * L.region_bytes; };
    LaneRegion* rinfo = rinfo_sm[w];
    uint32_t* meta = meta_sm[w];            // slot -> (region << 29) | child index in its parent
    uint8_t* batch = smp<uint8_t>(rg(0), L.o_batch);
    // byte / child / round counters: per warp in shared memory (kept out of the registers the
    // parent loop holds); each flush adds its batch's warp sums
    __shared__ unsigned long long stats_sm[8][4];
    unsigned long long* wstats = stats_sm[w];
    if (lane < 4) wstats[lane] = 0;
    __syncwarp();
    uint32_t nb = 0, held = 0, cur = 0;     // children in the batch, regions they come from
    auto flush = [&]() {
        uint64_t b_stage = 0, b_hbm = 0, n_rounds = 0;
        if (lane < nb) {
            const uint32_t m = meta[lane], r = m >> 29, idx = m & 0x1FFFFFFFu;
            const LaneRegion ri = rinfo[r];
            char* rs = rg(r);
            const DevRule& R = *smp<DevRule>(rs, L.o_rule);
            const Parent pa{ri.ne, ri.nocc, ri.nvp};
            const uint8_t* slot = batch + lane * L.SB;
            WlInfo info;
            const uint64_t h = lane_wl<kLaneVMax, kLaneNMax>(L, rs, pa, R, slot, info);
            const uint32_t e = ri.ev0 + idx;
            const uint32_t coff = ri.cons0 + idx * R.n_lhs;
            const uint32_t pid = ri.prod0 + idx * R.n_rhs;
            const uint32_t* peid = smp<uint32_t>(rs, L.o_peid);
            P.ev_in[e] = ri.sid;
            P.ev_rule[e] = ri.rule_g;
            P.ev_coff[e] = coff;
            P.ev_prod[e] = pid;
            P.ev_fresh[e] = ri.fresh0 + idx * R.n_fresh;
            P.ev_hash[e] = h;
            P.ev_nv[e] = info.nv;
            for (uint32_t k = 0; k < R.n_lhs; ++k) P.ev_cons[coff + k] = peid[slot[k]];
            P.ev_bmask[e] = branch_mask(R.n_lhs, pa.ne, slot);
            for (uint32_t k = 0; k < R.n_rhs; ++k) P.edge_creator[pid + k] = e;
            slot_insert(P, ri.table_off, ri.table_mask, h, e);
            const uint64_t k = R.n_lhs, rr = R.n_rhs;
            const uint32_t nec = pa.ne - R.n_lhs + R.n_rhs;
            b_stage += 4 * k + 8;
            b_stage += 4ull * pa.ne + 4ull * nec + 4ull * R.rhs_total + 12 * rr + 16 + 4 * k + 4 * rr;
            b_stage += 5ull * info.nocc + 8ull * info.nv +
                       uint64_t(info.rounds) * (8ull * info.nbr + 5ull * info.nocc + 16ull * info.nv) +
                       8ull * info.nv + 8ull * info.nocc;
            b_stage += 16;
            b_hbm += 20 + 8 + 8 * k + 4 * rr + 16;
            n_rounds += info.rounds;
        }
        b_stage = warp_sum64(b_stage);
        b_hbm = warp_sum64(b_hbm);
        n_rounds = warp_sum64(n_rounds);
        if (lane == 0) {
            wstats[0] += b_stage;
            wstats[1] += b_hbm;
            wstats[2] += nb;
            wstats[3] += n_rounds;
        }
        __syncwarp();
        nb = 0;
        held = 0;
    };
    WarpWork q;
    while (true) {
        const uint32_t u = q.next(&A.work[1]);
        if (u >= A.f_end - A.f_begin) break;
        const uint32_t f = frontier_at(A, A.f_begin + u);
        const uint8_t fm = A.fmode[f];
        if (!(fm & 1u)) continue;
        const uint32_t rn = A.counts[f];              // single-rule evolutions: item = f
        const uint32_t sid = A.frontier[f];
        const uint32_t evo = P.st_evo[sid];
        const DevEvo ev = P.evos[evo];
        if (rn == 0 || ev.rule_count == 0) {   // nothing to build: count what the join reads
            if (lane == 0) {
                const uint64_t ne = P.st_ne[sid], nocc = P.st_nocc[sid];
                wstats[1] += 4 * (ne + (ne + 3) / 4 + nocc) + 20;
                wstats[0] += 4 * ne + 4 * nocc;
            }
            continue;
        }
        if ((held >> cur) & 1u) flush();             // the region still feeds the batch
        char* sm = rg(cur);
        const Parent pa = load_parent(P, L, sm, sid);
        build_parent_csr(L, sm, pa);
        load_rule(sm, L, &P.rules[ev.rule_begin]);
        const DevRule& R = *smp<DevRule>(sm, L.o_rule);
        if (lane == 0) {
            wstats[1] += 4ull * (pa.ne + (pa.ne + 3) / 4 + pa.nocc) + 20;
            wstats[0] += 4ull * pa.ne + 4ull * pa.nocc;
            LaneRegion ri;
            ri.sid = sid;
            ri.ev0 = A.ev_base + A.item_ev[f];
            ri.cons0 = A.cons_base + A.item_cons[f];
            ri.prod0 = A.prod_base + A.item_prod[f];
            ri.fresh0 = A.fresh_base + A.item_fresh[f];
            ri.rule_g = ev.rule_begin;
            ri.ne = pa.ne;
            ri.nocc = pa.nocc;
            ri.nvp = pa.nvp;
            ri.table_off = ev.table_off;
            ri.table_mask = ev.table_mask;
            rinfo[cur] = ri;
        }
        __syncwarp();
        Fwd fwd;
        fwd.on = false;
        if constexpr (kFwd) fwd = fwd_prepare(P, A, L, sm, R, ev, pa, sid, (fm & 2u) != 0);
        if (kWalk && !fwd.on && pa.ne <= kLaneEMax && R.n_lhs <= kLaneJoinLhs && rn <= L.MCAP) {
            uint32_t* mlist = smp<uint32_t>(rg(0), L.o_mlist);   // the warp's one match list
            const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
            const uint16_t* vloc = smp<uint16_t>(sm, L.o_vloc);
            uint32_t total = 0;
            for (uint32_t b = 0; b < pa.ne; b += 32) {
                const uint32_t e0 = b + lane;
                const uint32_t c = e0 < pa.ne ? lane_walk(L, sm, R, pa, e0, [](uint32_t) {}) : 0u;
                const uint32_t inc = warp_incl_scan(c);
                uint32_t wpos = total + inc - c;
                if (c) lane_walk(L, sm, R, pa, e0, [&](uint32_t pk) {
                    if (wpos < L.MCAP) mlist[wpos] = pk;
                    ++wpos;
                });
                total += __shfl_sync(0xFFFFFFFFu, inc, 31);
            }
            __syncwarp();
            if (total != rn) {
                if (lane == 0) atomicOr(P.err, kErrJoinCount);
                continue;
            }
            for (uint32_t i0 = 0; i0 < rn;) {
                const uint32_t take = min(rn - i0, 32u - nb);
                if (lane < take) {
                    const uint32_t i = i0 + lane, sl = nb + lane;
                    uint8_t* slot = batch + sl * L.SB;
                    const uint32_t pk = mlist[i];
                    uint16_t bv[kMaxVars];
                    for (uint32_t k = 0; k < R.n_lhs; ++k) {
                        const uint32_t pos = (pk >> (8u * k)) & 0xFFu;
                        slot[k] = static_cast<uint8_t>(pos);
                        const uint32_t vo = pevo[pos];
                        for (uint32_t qq = 0; qq < R.lhs_ar[k]; ++qq)
                            bv[R.lhs_vars[R.lhs_off[k] + qq]] = vloc[vo + qq];
                    }
                    for (uint32_t t = 0; t < R.rhs_total; ++t) {
                        const uint32_t var = R.rhs_vars[t];
                        slot[R.n_lhs + t] = static_cast<uint8_t>(((R.new_mask >> var) & 1u)
                                                                 ? pa.nvp + R.fresh_rank[var]
                                                                 : bv[var]);
                    }
                    meta[sl] = (cur << 29) | i;
                }
                __syncwarp();
                nb += take;
                i0 += take;
                held |= 1u << cur;
                if (nb == 32) flush();
            }
        } else {
            const uint16_t* match = smp<uint16_t>(sm, L.o_match);
            const uint16_t* bind = smp<uint16_t>(sm, L.o_bind);
            uint32_t idx = 0;
            auto on_match = [&](uint32_t nm) {
                uint8_t* slot = batch + nb * L.SB;
                if (lane < R.n_lhs) slot[lane] = static_cast<uint8_t>(match[lane]);
                for (uint32_t t = lane; t < R.rhs_total; t += 32) {
                    const uint32_t var = R.rhs_vars[t];
                    slot[R.n_lhs + t] = static_cast<uint8_t>(((nm >> var) & 1u) ? bind[var]
                                                             : pa.nvp + R.fresh_rank[var]);
                }
                if (lane == 0) meta[nb] = (cur << 29) | idx;
                __syncwarp();
                ++idx;
                ++nb;
                held |= 1u << cur;
                if (nb == 32) flush();
            };
            if constexpr (kFwd) enumerate_matches(P, L, sm, R, pa, fwd, on_match);
            else warp_join(L, sm, R, pa, R.sched, -1, on_match);
        }
        cur = cur + 1 == kReg ? 0u : cur + 1;
    }
    if (nb) flush();
    __syncwarp();
    if (lane == 0 && wstats[1]) {
        atomicAdd(&P.stats[0], wstats[0]);
        atomicAdd(&P.stats[1], wstats[1]);
        atomicAdd(&P.stats[2], wstats[2]);
        atomicAdd(&P.stats[3], wstats[3]);
    }
}

// ------------------------------------------------------------------------------------------
// Result finalisation for many evolutions at once. Their states (and events, pairs) are listed
// back to back, evolution after evolution; bases[k] is where evolution k's run starts (K + 1
// entries). Every output array of evolution k lives in its own section of one staging block:
// sec[k * kArr + a] is the byte offset of array a (hgx_array order). Local ids restart at 0 per
// evolution; a global id belongs to one evolution, so one global -> local map serves them all.
// ------------------------------------------------------------------------------------------
constexpr uint32_t kArr = 14;

__device__ __forceinline__ uint32_t seg_of(const uint32_t* bases, uint32_t K, uint32_t i) {
    uint32_t a = 0, b = K;   // largest k < K with bases[k] <= i
    while (b - a > 1) {
        const uint32_t m = (a + b) >> 1;
        if (bases[m] <= i) a = m; else b = m;
    }
    return a;
}

template <class T>
__device__ __forceinline__ T* sec_ptr(uint8_t* stage, const uint64_t* sec, uint32_t k, uint32_t a) {
    return reinterpret_cast<T*>(stage + sec[uint64_t(k) * kArr + a]);
}

// out[i] = rstart[r] + (i - rcum[r]) over nr ranges with exclusive prefix rcum (ids of many ranges).
__global__ void k_expand_ranges(const uint64_t* rstart, const uint64_t* rcum, uint32_t nr, uint64_t n,
                                uint32_t* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t a = 0, b = nr;
        while (b - a > 1) {
            const uint32_t m = (a + b) >> 1;
            if (rcum[m] <= i) a = m; else b = m;
        }
        out[i] = static_cast<uint32_t>(rstart[a] + (i - rcum[a]));
    }
}

__global__ void k_map_multi(const uint32_t* ids, uint32_t n, const uint32_t* bases, uint32_t K,
                            uint32_t* map) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        map[ids[i]] = i - bases[seg_of(bases, K, i)];
}

// States: hash and depth into their sections (stage set), or edge / occurrence counts for the
// CSR scans (stage null).
__global__ void k_fin_states_multi(DevPtrs P, const uint32_t* sids, uint32_t n, const uint32_t* sb,
                                   uint32_t K, uint8_t* stage, const uint64_t* sec, uint32_t* ne,
                                   uint32_t* nocc) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = sids[i];
        if (stage) {
            const uint32_t k = seg_of(sb, K, i), j = i - sb[k];
            sec_ptr<uint64_t>(stage, sec, k, 0)[j] = P.st_hash[s];
            sec_ptr<uint32_t>(stage, sec, k, 1)[j] = P.st_depth[s];
        } else {
            ne[i] = P.st_ne[s];
            nocc[i] = P.st_nocc[s];
        }
    }
}

// The CSR offsets of one array kind relative to each evolution's start (entries 0..n_k).
__global__ void k_fin_offsets_multi(const uint32_t* scan, uint32_t n, const uint32_t* bases,
                                    uint32_t K, uint8_t* stage, const uint64_t* sec, uint32_t arr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n + K; i += gridDim.x * blockDim.x) {
        // i < n: entry j of its evolution; i >= n: the closing entry of evolution i - n
        uint32_t k, j, at;
        if (i < n) { k = seg_of(bases, K, i); j = i - bases[k]; at = i; }
        else { k = i - n; j = bases[k + 1] - bases[k]; at = bases[k + 1]; }
        sec_ptr<uint32_t>(stage, sec, k, arr)[j] = scan[at] - scan[bases[k]];
    }
}

__global__ void k_fin_records_multi(DevPtrs P, const uint32_t* sids, uint32_t n, const uint32_t* sb,
                                    uint32_t K, const uint32_t* eoff, const uint32_t* voff,
                                    uint8_t* stage, const uint64_t* sec, int with_ids) {
    const uint32_t lane = lane_id();
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t s = sids[i], k = seg_of(sb, K, i);
        const uint32_t e0 = eoff[i] - eoff[sb[k]], v0 = voff[i] - voff[sb[k]];
        uint32_t* oids = sec_ptr<uint32_t>(stage, sec, k, 9);
        uint8_t* oar = sec_ptr<uint8_t>(stage, sec, k, 10);
        uint32_t* overts = sec_ptr<uint32_t>(stage, sec, k, 12);
        const uint32_t ne = P.st_ne[s], nocc = P.st_nocc[s], aw = (ne + 3) >> 2;
        const uint32_t* rec = P.arena + P.st_off[s];
        for (uint32_t t = lane; t < ne; t += 32) {
            if (with_ids) oids[e0 + t] = rec[t];
            oar[e0 + t] = static_cast<uint8_t>(rec[ne + (t >> 2)] >> ((t & 3u) * 8u));
        }
        for (uint32_t t = lane; t < nocc; t += 32) overts[v0 + t] = rec[ne + aw + t];
    }
}

// Events. pass 0: consumed and causal counts (for the scans); pass 1: tuples, consumed lists,
// produced ranges, causal triples and signatures into their evolutions' sections.
__global__ void k_fin_events_multi(DevPtrs P, const uint32_t* eids, uint32_t n, const uint32_t* eb,
                                   uint32_t K, const uint32_t* rule_begin, const uint32_t* smap,
                                   const uint32_t* emap, uint32_t* ccount, uint32_t* kcount,
                                   const uint32_t* coff, const uint32_t* koff, uint8_t* stage,
                                   const uint64_t* sec, int pass, int causal, int sig) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = eids[i];
        const uint32_t r = P.ev_rule[e];
        const DevRule& R = P.rules[r];
        const uint32_t co = P.ev_coff[e];
        if (!pass) {
            uint32_t c = 0;
            for (uint32_t j = 0; j < R.n_lhs; ++j) c += P.ev_cprod[co + j] != kNone ? 1u : 0u;
            ccount[i] = R.n_lhs;
            kcount[i] = causal ? c : 0u;
            continue;
        }
        const uint32_t k = seg_of(eb, K, i), li = i - eb[k];
        const uint32_t in = P.ev_in[e];
        uint32_t* tup = sec_ptr<uint32_t>(stage, sec, k, 2);
        tup[4 * li] = smap[in];
        tup[4 * li + 1] = smap[P.ev_out[e]];
        tup[4 * li + 2] = r - rule_begin[k];
        tup[4 * li + 3] = P.st_depth[in] + 1;
        uint32_t* prod = sec_ptr<uint32_t>(stage, sec, k, 7);
        prod[2 * li] = P.ev_prod[e];
        prod[2 * li + 1] = R.n_rhs;
        if (sig) sec_ptr<uint64_t>(stage, sec, k, 13)[li] = P.ev_sig[e];
        uint32_t* cons = sec_ptr<uint32_t>(stage, sec, k, 6);
        uint32_t* tri = sec_ptr<uint32_t>(stage, sec, k, 3);
        const uint32_t c0 = coff[i] - coff[eb[k]];
        uint32_t w = koff[i] - koff[eb[k]];
        for (uint32_t j = 0; j < R.n_lhs; ++j) {
            const uint32_t c = P.ev_cons[co + j];
            cons[c0 + j] = c;
            const uint32_t p = P.ev_cprod[co + j];
            if (!causal || p == kNone) continue;
            tri[3 * w] = emap[p];
            tri[3 * w + 1] = li;
            tri[3 * w + 2] = c;
            ++w;
        }
    }
}

// Branchial pairs of every listed evolution: nr ranges of the pair array (exclusive prefix rcum);
// evolution k owns the pair run [pb[k], pb[k+1]) of the concatenation.
__global__ void k_fin_pairs_multi(const uint32_t* pairs, const uint64_t* rstart, const uint64_t* rcum,
                                  uint32_t nr, uint64_t n, const uint32_t* pb, uint32_t K,
                                  const uint32_t* emap, uint8_t* stage, const uint64_t* sec) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t a = 0, b = nr;
        while (b - a > 1) {
            const uint32_t m = (a + b) >> 1;
            if (rcum[m] <= i) a = m; else b = m;
        }
        const uint64_t g = rstart[a] + (i - rcum[a]);
        const uint32_t k = seg_of(pb, K, static_cast<uint32_t>(i));
        uint32_t* out = sec_ptr<uint32_t>(stage, sec, k, 4);
        const uint64_t li = i - pb[k];
        out[2 * li] = emap[pairs[2 * g]];
        out[2 * li + 1] = emap[pairs[2 * g + 1]];
    }
}

// A single zero entry per evolution (the offset arrays of state records not kept).
__global__ void k_fin_zero_multi(uint8_t* stage, const uint64_t* sec, uint32_t K, uint32_t arr) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        sec_ptr<uint32_t>(stage, sec, k, arr)[0] = 0;
}

// Values of a scanned array at every evolution boundary (K + 1 of them), for the host.
__global__ void k_fin_bounds(const uint32_t* scan, const uint32_t* bases, uint32_t K, uint32_t* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= K; k += gridDim.x * blockDim.x)
        out[k] = scan[bases[k]];
}

// Each frontier state's event range (its matches, in canonical order), for its children's
// match forwarding. Single-rule evolutions only (item f * R of the state).

// Roots: count WL classes (first arrival of each hash) and states per evolution.
__global__ void k_root_counts(DevPtrs P, const uint32_t* sids, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t sid = sids[i];
        const uint32_t evo = P.st_evo[sid];
        const uint32_t w = table_lookup(P, P.evos[evo], P.st_hash[sid]);
        if (w == P.st_event[sid]) atomicAdd(&P.evo_classes[evo], 1ull);
        atomicAdd(&P.evo_states[evo], 1ull);
    }
}

// Move one evolution's table into a larger region (values are already the minimum arrival).
__global__ void k_rehash(unsigned long long* keys, uint32_t* vals, uint64_t old_off,
                         uint64_t old_mask, uint64_t new_off, uint64_t new_mask, uint32_t* err) {
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s <= old_mask + 1;
         s += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = vals[old_off + s];
        if (s == old_mask + 1) {
            if (v != kNone) atomicMin(&vals[new_off + new_mask + 1], v);
            continue;
        }
        const unsigned long long k = keys[old_off + s];
        if (k == 0ull) continue;
        uint64_t slot = smix(k) & new_mask;
        bool done = false;
        for (uint64_t probe = 0; probe <= new_mask && !done; ++probe) {
            unsigned long long* kp = &keys[new_off + slot];
            unsigned long long cur = atomicCAS(kp, 0ull, k);
            if (cur == 0ull || cur == k) {
                atomicMin(&vals[new_off + slot], v);
                done = true;
            }
            slot = (slot + 1) & new_mask;
        }
        if (!done) atomicOr(err, kErrTableFull);
    }
}

// Is the child the first arrival of its WL class? (winner stored in ev_out until resolved)
__global__ void k_select(DevPtrs P, LevelArgs A, uint32_t t_begin, uint32_t t_end) {
    for (uint32_t t = t_begin + blockIdx.x * blockDim.x + threadIdx.x; t < t_end;
         t += gridDim.x * blockDim.x) {
        const uint32_t e = A.ev_base + t;
        const uint32_t evo = P.st_evo[P.ev_in[e]];
        const uint32_t w = table_lookup(P, P.evos[evo], P.ev_hash[e]);
        P.ev_out[e] = w;
        A.flag_new[t] = (w == e) ? 1u : 0u;
    }
}

// k_select over the events of the frontier ranges in A.frng (a warp per state); the new classes
// found are added to evo_new[evolution].
__global__ void k_select_list(DevPtrs P, LevelArgs A, uint32_t n, unsigned long long* evo_new) {
    const uint32_t lane = lane_id();
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t f = frontier_at(A, i);
        const uint32_t lo = A.item_ev[f * A.rules_stride], hi = A.item_ev[(f + 1) * A.rules_stride];
        const uint32_t evo = P.st_evo[A.frontier[f]];
        const DevEvo ev = P.evos[evo];
        uint32_t c = 0;
        for (uint32_t t = lo + lane; t < hi; t += 32) {
            const uint32_t e = A.ev_base + t;
            const uint32_t w = table_lookup(P, ev, P.ev_hash[e]);
            P.ev_out[e] = w;
            A.flag_new[t] = (w == e) ? 1u : 0u;
            c += (w == e) ? 1u : 0u;
        }
        c = warp_sum32(c);
        if (lane == 0 && c) atomicAdd(&evo_new[evo], static_cast<unsigned long long>(c));
    }
}

// Events of frontier states that a capped level never built (they all come after the
// evolution's cut): give them in-range ids so the per-event kernels see ordinary events that the
// cap dropped (k_rep marks them not kept).
__global__ void k_void(DevPtrs P, LevelArgs A, uint32_t n) {
    const uint32_t lane = lane_id();
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t f = frontier_at(A, i);
        const uint32_t sid = A.frontier[f];
        const DevEvo ev = P.evos[P.st_evo[sid]];
        for (uint32_t r = 0; r < A.rules_stride && r < ev.rule_count; ++r) {
            const uint32_t item = f * A.rules_stride + r;
            const uint32_t lo = A.item_ev[item], cnt = A.item_ev[item + 1] - lo;
            if (!cnt) continue;
            const DevRule& R = P.rules[ev.rule_begin + r];
            const uint32_t cons0 = A.cons_base + A.item_cons[item];
            const uint32_t prod0 = A.prod_base + A.item_prod[item];
            const uint32_t fresh0 = A.fresh_base + A.item_fresh[item];
            for (uint32_t idx = lane; idx < cnt; idx += 32) {
                const uint32_t e = A.ev_base + lo + idx;
                const uint32_t coff = cons0 + idx * R.n_lhs, pid = prod0 + idx * R.n_rhs;
                P.ev_in[e] = sid;
                P.ev_rule[e] = ev.rule_begin + r;
                P.ev_coff[e] = coff;
                P.ev_prod[e] = pid;
                P.ev_fresh[e] = fresh0 + idx * R.n_fresh;
                P.ev_hash[e] = 0;
                P.ev_out[e] = kNone;
                for (uint32_t k = 0; k < R.n_lhs; ++k) P.ev_cons[coff + k] = 0;   // edge 0 exists
                P.ev_bmask[e] = kMaskDropped;   // never kept
                for (uint32_t k = 0; k < R.n_rhs; ++k) P.edge_creator[pid + k] = e;
                A.flag_new[lo + idx] = 0;
            }
        }
    }
}

// State cap: the first event of an evolution that would take it past max_states cuts the level
// there; that event and every later one of the evolution in this level are dropped and the
// evolution stops expanding.
__global__ void k_cut(DevPtrs P, LevelArgs A) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A.n_events;
         t += gridDim.x * blockDim.x) {
        const uint32_t e = A.ev_base + t;
        const uint32_t evo = P.st_evo[P.ev_in[e]];
        const DevEvo& ev = P.evos[evo];
        if (!ev.max_states) continue;
        const uint32_t first = P.evo_first_ev[evo] - A.ev_base;
        if (ev.quotient) {
            if (!A.flag_new[t]) continue;
            const uint64_t rank = A.scan_new[t] - A.scan_new[first] + 1;
            const uint64_t have = P.evo_classes[evo];
            if (have + rank > ev.max_states) atomicMin(&P.evo_cut[evo], e);
        } else {
            const uint64_t rank = t - first + 1;
            if (P.evo_states[evo] + rank > ev.max_states) atomicMin(&P.evo_cut[evo], e);
        }
    }
}

__global__ void k_rep(DevPtrs P, LevelArgs A) {
    for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < A.n_events; t0 += gridDim.x * blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        const bool valid = t < A.n_events;
        uint32_t evo = 0;
        bool kept = false, fresh = false, rep = false;
        if (valid) {
            const uint32_t e = A.ev_base + t;
            const uint32_t sid = P.ev_in[e];
            evo = P.st_evo[sid];
            const DevEvo& ev = P.evos[evo];
            const uint32_t cut = P.evo_cut[evo];
            kept = e < cut;
            fresh = kept && A.flag_new[t];
            rep = kept && (ev.quotient ? fresh : true);
            const bool front = rep && (P.st_depth[sid] + 1 < ev.steps) && cut == kNone;
            P.ev_kept[e] = kept ? 1 : 0;
            if (!kept && P.ev_bmask[e]) P.ev_bmask[e] = kMaskDropped;
            A.flag_rep[t] = rep ? 1u : 0u;
            A.flag_front[t] = front ? 1u : 0u;
            if (e == cut) P.evo_stopped[evo] = 1;
        }
        warp_count(P.evo_classes, evo, fresh);
        warp_count(P.evo_states, evo, rep);
    }
}

// Representatives become states (ids in event order); eligible ones form the next frontier.
__global__ void k_assign(DevPtrs P, LevelArgs A) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A.n_events;
         t += gridDim.x * blockDim.x) {
        const uint32_t e = A.ev_base + t;
        const bool rep = A.flag_rep[t + 1] != A.flag_rep[t];
        if (!rep) continue;
        const uint32_t j = A.flag_rep[t];
        const uint32_t sid = A.state_base + j;
        const uint32_t in = P.ev_in[e];
        P.state_of_arrival[e] = sid;
        A.new_state_event[j] = e;
        P.st_event[sid] = e;
        P.st_evo[sid] = P.st_evo[in];
        P.st_depth[sid] = P.st_depth[in] + 1;
        P.st_hash[sid] = P.ev_hash[e];
        if (A.flag_front[t + 1] != A.flag_front[t]) A.next_frontier[A.flag_front[t]] = sid;
    }
}

// Also counts each evolution's causal triples (the kept events' consumed edges that have a
// producer; the level's producers are final here, after k_cprod and k_tr).
__global__ void k_outstate(DevPtrs P, LevelArgs A) {
    for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < A.n_events; t0 += gridDim.x * blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        uint32_t evo = 0, nc = 0;
        if (t < A.n_events) {
            const uint32_t e = A.ev_base + t;
            if (!P.ev_kept[e]) {
                P.ev_out[e] = kNone;
            } else {
                evo = P.st_evo[P.ev_in[e]];
                const bool rep = A.flag_rep[t + 1] != A.flag_rep[t];
                if (rep || !P.evos[evo].quotient) {
                    P.ev_out[e] = P.state_of_arrival[e];
                } else {
                    const uint32_t w = P.ev_out[e];
                    if (w == kNone) { atomicOr(P.err, kErrTableFull); P.ev_out[e] = kNone; }
                    else P.ev_out[e] = P.state_of_arrival[w];
                }
                const uint32_t co = P.ev_coff[e], k = P.rules[P.ev_rule[e]].n_lhs;
                for (uint32_t i = 0; i < k; ++i) nc += P.ev_cprod[co + i] != kNone ? 1u : 0u;
            }
        }
        // per evolution, one atomic per warp
        const bool live = nc != 0;
        const uint32_t act = __ballot_sync(0xFFFFFFFFu, live);
        if (live) {
            const uint32_t peers = __match_any_sync(act, evo);
            uint32_t sum = nc;
            for (uint32_t m = peers & ~(1u << lane_id()); m; m &= m - 1)
                sum += __shfl_sync(peers, nc, __ffs(m) - 1);
            if (lane_id() == static_cast<uint32_t>(__ffs(peers) - 1))
                atomicAdd(&P.evo_causal[evo], static_cast<unsigned long long>(sum));
        }
    }
}

// Event canonicalisation (Hypergraph::create_event, hypergraph/src/hypergraph.cpp:449-500): the
// signature of every kept event of the level from its input and output states' WL hashes, the
// step of the output's canonical state -- the first state of its class, whose arrival the dedup
// table holds (hypergraph.cpp:362-377) -- and its rule; pass 0 inserts it into the evolution's
// signature table (smallest event id wins, so across levels the first event in canonical order is
// the canonical one); pass 1 counts the winners per evolution.
__global__ void k_evsig(DevPtrs P, LevelArgs A, int pass) {
    for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < A.n_events; t0 += gridDim.x * blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        uint32_t evo = 0;
        bool win = false;
        if (t < A.n_events) {
            const uint32_t e = A.ev_base + t;
            if (P.ev_kept[e]) {
                const uint32_t in = P.ev_in[e];
                evo = P.st_evo[in];
                const DevEvo& ev = P.evos[evo];
                if (pass == 0) {
                    const uint32_t first = table_lookup(P, ev, P.ev_hash[e]);
                    const uint32_t fin = first == kNone ? kNone : P.ev_in[first];
                    const uint32_t step = fin == kNone ? 0u : P.st_depth[fin] + 1;
                    const uint64_t sig = event_signature(A.ev_keys, P.st_hash[in], P.ev_hash[e],
                                                         step, P.ev_rule[e] - ev.rule_begin);
                    P.ev_sig[e] = sig;
                    slot_insert(P, ev.sig_off, ev.sig_mask, sig, e);
                } else {
                    win = slot_lookup(P, ev.sig_off, ev.sig_mask, P.ev_sig[e]) == e;
                }
            }
        }
        if (pass == 1) warp_count(P.evo_sigs, evo, win);
    }
}

// Inclusive scan inside segments of S lanes (S = 32: the whole warp).
template <uint32_t S>
__device__ __forceinline__ uint32_t seg_incl_scan(uint32_t x) {
#pragma unroll
    for (uint32_t d = 1; d < S; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d, S);
        if ((lane_id() & (S - 1)) >= d) x += y;
    }
    return x;
}

// Write the edge record of every new state: parent edges minus consumed, then produced.
// Groups of 32 new states per warp share one arena reservation and one level-maximum update;
// the group's states are then written 32 / S at a time, one per segment of S lanes (lanes =
// parent edges), S chosen on the host from the level's largest parent (8, 16 or 32 edges per
// pass), so a small parent does not leave most of the warp idle.
// Held to 64 registers (4 blocks per SM; no spills): C2 materialise 0.99 -> 0.87 ms.
template <uint32_t S>
__global__ void __launch_bounds__(256, 4) k_materialize(DevPtrs P, LevelArgs A, uint32_t n_new) {
    constexpr uint32_t G = 32 / S;
    __shared__ uint32_t bind_sm[8][G][kMaxVars];
    __shared__ uint32_t cons_sm[8][G][kMaxPatternEdges];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t seg = lane / S, sl = lane & (S - 1);
    const uint32_t segbits = S == 32 ? 0xFFFFFFFFu : ((1u << S) - 1u);
    uint32_t* bind = bind_sm[w][seg];
    uint32_t* cons = cons_sm[w][seg];
    // groups of 32 new states per warp: record sizes by lane, one arena reservation per group
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g * 32ull < n_new;
         g += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t jl = g * 32 + lane;
        uint32_t words = 0, gne = 0, gnocc = 0;
        // lane k loads state k's event, parent and rule once; the loop below takes them by
        // shuffle instead of repeating the chain of dependent loads per state
        uint32_t e_l = 0, f_l = 0, r_l = 0, pne_l = 0, pnocc_l = 0, coff_l = 0, pid_l = 0, fid_l = 0;
        unsigned long long poff_l = 0;
        if (jl < n_new) {
            e_l = A.new_state_event[jl];
            f_l = P.ev_in[e_l];
            r_l = P.ev_rule[e_l];
            coff_l = P.ev_coff[e_l];
            pid_l = P.ev_prod[e_l];
            fid_l = P.ev_fresh[e_l];
            const DevRule& R = P.rules[r_l];
            pne_l = P.st_ne[f_l];
            pnocc_l = P.st_nocc[f_l];
            poff_l = P.st_off[f_l];
            gne = pne_l - R.n_lhs + R.n_rhs;
            gnocc = pnocc_l - R.lhs_total + R.rhs_total;
            words = gne + ((gne + 3) >> 2) + gnocc;
            P.st_nv[A.state_base + jl] = P.ev_nv[e_l];
        }
        const uint32_t inc = warp_incl_scan(words);
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
        gne = warp_max32(gne);
        gnocc = warp_max32(gnocc);
        unsigned long long base = 0;
        if (lane == 0) {
            base = atomicAdd(P.arena_top, static_cast<unsigned long long>(total));
            atomicMax(&A.level_max[0], gne);
            atomicMax(&A.level_max[1], gnocc);
        }
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base + total > P.arena_cap) {
            if (lane == 0) atomicOr(P.err, kErrArenaFull);
            continue;
        }
        const unsigned long long my_off = base + inc - words;
        const uint32_t cnt = min(32u, n_new - g * 32);
        for (uint32_t k0 = 0; k0 < cnt; k0 += G) {
            const uint32_t k = k0 + seg;               // this segment's state in the group
            const bool act = k < cnt;
            const uint32_t src = act ? k : 0u;
            const uint32_t j = g * 32 + k;
            const unsigned long long off = __shfl_sync(0xFFFFFFFFu, my_off, src);
            const uint32_t sid = A.state_base + j;
            const DevRule& R = P.rules[__shfl_sync(0xFFFFFFFFu, r_l, src)];
            // every lane takes part in every shuffle (a full-mask shuffle that some lanes skip
            // never completes); inactive segments then zero what they took
            const uint32_t pne_s = __shfl_sync(0xFFFFFFFFu, pne_l, src);
            const uint32_t pne = act ? pne_s : 0u;
            const uint32_t pnocc = __shfl_sync(0xFFFFFFFFu, pnocc_l, src);
            const uint32_t coff = __shfl_sync(0xFFFFFFFFu, coff_l, src);
            const uint32_t* prec = P.arena + __shfl_sync(0xFFFFFFFFu, poff_l, src);
            const uint32_t pid = __shfl_sync(0xFFFFFFFFu, pid_l, src);
            const uint32_t fid = __shfl_sync(0xFFFFFFFFu, fid_l, src);
            const uint32_t paw = (pne + 3) >> 2;
            const uint32_t ne = act ? pne - R.n_lhs + R.n_rhs : 0u;
            const uint32_t nocc = act ? pnocc - R.lhs_total + R.rhs_total : 0u;
            const uint32_t aw = (ne + 3) >> 2;
            uint32_t* rec = P.arena + off;
            uint8_t* rar = reinterpret_cast<uint8_t*>(rec + ne);
            uint32_t* rv = rec + ne + aw;
            if (act)
                for (uint32_t t = sl; t < R.n_lhs; t += S) cons[t] = P.ev_cons[coff + t];
            if (act)
                for (uint32_t t = sl; t < aw; t += S) rec[ne + t] = 0;   // arity padding bytes
            __syncwarp();
            // kept parent edges; a consumed edge binds its pattern edge's variables instead
            uint32_t pne_max = pne;
#pragma unroll
            for (uint32_t d = S; d < 32; d <<= 1) pne_max = max(pne_max, __shfl_xor_sync(0xFFFFFFFFu, pne_max, d));
            uint32_t run_e = 0, run_pv = 0, run_cv = 0;
            for (uint32_t b = 0; b < pne_max; b += S) {
                const uint32_t i = b + sl;
                uint32_t id = 0, a = 0, hit = kNone;
                if (i < pne) {
                    id = prec[i];
                    a = (prec[pne + (i >> 2)] >> ((i & 3u) * 8u)) & 0xFFu;
                    for (uint32_t k2 = 0; k2 < R.n_lhs; ++k2)
                        if (cons[k2] == id) hit = k2;
                }
                const bool keep = i < pne && hit == kNone;
                const uint32_t pinc = seg_incl_scan<S>(a);
                const uint32_t ka = keep ? a : 0u;
                const uint32_t kinc = seg_incl_scan<S>(ka);
                const uint32_t bal = (__ballot_sync(0xFFFFFFFFu, keep) >> (seg * S)) & segbits;
                const uint32_t sv = run_pv + pinc - a;
                if (keep) {
                    const uint32_t c = run_e + __popc(bal & ((1u << sl) - 1u));
                    rec[c] = id;
                    rar[c] = static_cast<uint8_t>(a);
                    const uint32_t dst = run_cv + kinc - ka;
                    for (uint32_t q = 0; q < a; ++q) rv[dst + q] = prec[pne + paw + sv + q];
                } else if (hit != kNone) {
                    for (uint32_t q = 0; q < a; ++q)
                        bind[R.lhs_vars[R.lhs_off[hit] + q]] = prec[pne + paw + sv + q];
                }
                run_e += __popc(bal);
                run_pv += __shfl_sync(0xFFFFFFFFu, pinc, S - 1, S);
                run_cv += __shfl_sync(0xFFFFFFFFu, kinc, S - 1, S);
            }
            __syncwarp();
            // produced edges
            if (act) {
                for (uint32_t k2 = sl; k2 < R.n_rhs; k2 += S) {
                    rec[run_e + k2] = pid + k2;
                    rar[run_e + k2] = R.rhs_ar[k2];
                }
                for (uint32_t t = sl; t < R.rhs_total; t += S) {
                    const uint32_t var = R.rhs_vars[t];
                    rv[run_cv + t] = ((R.new_mask >> var) & 1u) ? fid + R.fresh_rank[var] : bind[var];
                }
                if (sl == 0) {
                    P.st_off[sid] = off;
                    P.st_ne[sid] = ne;
                    P.st_nocc[sid] = nocc;
                }
            }
            __syncwarp();
        }
    }
}

// Branchial pairs (CausalGraph::record_branchial_overlaps, hypergraph/src/causal_graph.cpp:324-350):
// two kept events of the same input state that consumed a common edge, each unordered pair once
// as (a, b), a < b. The events of one input state are contiguous (they are numbered in frontier
// order). Pass 0 counts a's pairs into bcount[t]; pass 1 writes them at the scanned offset
// boff[t] in (a, then b) order.
//
// One event a (level index t) walking its successors until the input state changes: the form for
// states whose events carry no position masks (parents past 63 edges; the test compares edge ids).
template <bool kEmit>
__device__ void bpairs_walk(const DevPtrs& P, const LevelArgs& A, uint32_t t) {
    const uint32_t a = A.ev_base + t;
    const uint32_t end = A.ev_base + A.n_events;
    uint32_t cnt = 0;
    if (P.ev_kept[a]) {
        const uint32_t in = P.ev_in[a];
        const uint32_t na = P.rules[P.ev_rule[a]].n_lhs, ca0 = P.ev_coff[a];
        const unsigned long long ma = P.ev_bmask[a];
        uint32_t ca[kMaxPatternEdges];   // edge ids, for parents past the mask's 63 positions
        bool have_ca = false;
        uint32_t out = kEmit ? A.boff[t] : 0u;
        for (uint32_t c = a + 1; c < end && P.ev_in[c] == in; ++c) {
            const unsigned long long mc = P.ev_bmask[c];
            bool share = false;
            if (ma && mc) {
                // a consumed parent position in common (never with a dropped event's mask)
                share = (ma & mc) != 0ull;
            } else if (P.ev_kept[c]) {
                if (!have_ca) {
                    for (uint32_t k = 0; k < na; ++k) ca[k] = P.ev_cons[ca0 + k];
                    have_ca = true;
                }
                const uint32_t nc = P.rules[P.ev_rule[c]].n_lhs, cc0 = P.ev_coff[c];
                for (uint32_t k = 0; k < nc && !share; ++k) {
                    const uint32_t x = P.ev_cons[cc0 + k];
                    for (uint32_t m = 0; m < na; ++m) share |= (ca[m] == x);
                }
            }
            if (!share) continue;
            if (kEmit) reinterpret_cast<uint2*>(A.bpairs)[out++] = make_uint2(a, c);
            ++cnt;
        }
    }
    if (!kEmit) A.bcount[t] = cnt;
}

// Thread per event of the level whose parent carries no position masks (more than 63 edges; then
// none of its events has one): the per-event walk. The other events are k_bpairs'.
template <bool kEmit>
__global__ void k_bpairs_walk(DevPtrs P, LevelArgs A) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A.n_events; t += gridDim.x * blockDim.x)
        if (P.ev_bmask[A.ev_base + t] == 0ull) bpairs_walk<kEmit>(P, A, t);
}

// Warp per input state (frontier position f, events [item_ev[f R], item_ev[(f+1) R]) of the
// level) whose events carry position masks (a parent of at most 63 edges; a dropped event carries
// kMaskDropped): lane i holds the mask of event i of a 32-event tile and takes the masks of the
// later events from the other lanes by shuffles, so every pair test is one AND of registers.
template <bool kEmit>
__global__ void k_bpairs(DevPtrs P, LevelArgs A) {
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t R = A.rules_stride;
    for (uint32_t f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); f < A.n_frontier; f += warps) {
        const uint32_t g0 = A.item_ev[f * R];
        const uint32_t g1 = min(A.item_ev[(f + 1) * R], A.n_events);
        if (g1 <= g0) continue;
        const uint32_t k = g1 - g0;
        const uint32_t e0 = A.ev_base + g0;
        if (P.ev_bmask[e0] == 0ull) continue;   // no masks: k_bpairs_walk's
        for (uint32_t t0 = 0; t0 < k; t0 += 32) {
            const uint32_t i = t0 + lane;
            const bool mine = i < k;
            // a dropped event pairs with nothing
            const unsigned long long ma = (mine && P.ev_kept[e0 + i]) ? P.ev_bmask[e0 + i] : 0ull;
            uint32_t cnt = 0;
            uint32_t out = (kEmit && mine) ? A.boff[g0 + i] : 0u;
            for (uint32_t c0 = t0; c0 < k; c0 += 32) {
                const uint32_t ic = c0 + lane;
                const unsigned long long mine_c = ic < k ? P.ev_bmask[e0 + ic] : 0ull;
                const uint32_t jn = min(32u, k - c0);
                for (uint32_t j = 0; j < jn; ++j) {
                    const unsigned long long mc = __shfl_sync(0xFFFFFFFFu, mine_c, j);
                    if (c0 + j > i && (ma & mc) != 0ull) {
                        if (kEmit) reinterpret_cast<uint2*>(A.bpairs)[out++] = make_uint2(e0 + i, e0 + c0 + j);
                        ++cnt;
                    }
                }
            }
            if (!kEmit && mine) A.bcount[g0 + i] = cnt;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Result finalisation for a single-evolution run: local ids (roots hold the first `roots`
// arrival ids, so event e is local e - roots), the event tuples, the causal triples and the
// state records in state order, written into one staging buffer that is copied to the host once.
// ------------------------------------------------------------------------------------------
__global__ void k_fin_events(DevPtrs P, uint32_t roots, uint32_t n, uint32_t rule_begin,
                             uint32_t* tup, uint32_t* cons_off, uint32_t* prod, uint32_t c0) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = roots + i;
        const uint32_t in = P.ev_in[e];
        const uint32_t r = P.ev_rule[e];
        tup[4 * i] = in;
        tup[4 * i + 1] = P.ev_out[e];
        tup[4 * i + 2] = r - rule_begin;
        tup[4 * i + 3] = P.st_depth[in] + 1;
        cons_off[i] = P.ev_coff[e] - c0;
        prod[2 * i] = P.ev_prod[e];
        prod[2 * i + 1] = P.rules[r].n_rhs;
    }
}

// Causal triples of events first + i (i < n): pass 0 counts (into cnt[i]), pass 1 writes at the
// scanned offsets. Event ids are local (minus roots).
__global__ void k_fin_causal(DevPtrs P, uint32_t roots, uint32_t first, uint32_t n, uint32_t* cnt,
                             const uint32_t* off, uint32_t* out, int pass) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = first + i;
        const uint32_t co = P.ev_coff[e], k = P.rules[P.ev_rule[e]].n_lhs;
        uint32_t w = pass ? off[i] : 0u;
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t p = P.ev_cprod[co + j];
            if (p == kNone) continue;
            if (pass) {
                out[3 * w] = p - roots;
                out[3 * w + 1] = e - roots;
                out[3 * w + 2] = P.ev_cons[co + j];
            }
            ++w;
        }
        if (!pass) cnt[i] = w;
    }
}

__global__ void k_fin_shift(const uint32_t* in, uint64_t n, uint32_t sub, uint32_t* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = in[i] - sub;
}

// Warp per state s0 + s (s < n): its record's edge ids, arities and vertices at the scanned CSR
// offsets eoff[s] / voff[s].
__global__ void k_fin_states(DevPtrs P, uint32_t s0, uint32_t n, const uint32_t* eoff,
                             const uint32_t* voff, uint32_t* ids, uint8_t* ar, uint32_t* verts) {
    const uint32_t lane = lane_id();
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < n;
         s += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t ne = P.st_ne[s0 + s], nocc = P.st_nocc[s0 + s], aw = (ne + 3) >> 2;
        const uint32_t* rec = P.arena + P.st_off[s0 + s];
        const uint32_t e0 = eoff[s], v0 = voff[s];
        for (uint32_t i = lane; i < ne; i += 32) {
            if (ids) ids[e0 + i] = rec[i];   // null: the ids are not part of the result
            ar[e0 + i] = static_cast<uint8_t>(rec[ne + (i >> 2)] >> ((i & 3u) * 8u));
        }
        for (uint32_t j = lane; j < nocc; j += 32) verts[v0 + j] = rec[ne + aw + j];
    }
}

// Byte copy by the SMs (device to device, or device to page-locked host memory): copies the
// engine stream makes this way never queue on a copy engine behind the result copies of the copy
// stream. 16-byte words when both ends are 16-byte aligned, else bytes.
__global__ void k_copy_bytes(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint64_t n) {
    const uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0) {
        const uint64_t w = n / 16;
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(dst);
        for (uint64_t i = t; i < w; i += stride) d4[i] = s4[i];
        for (uint64_t i = w * 16 + t; i < n; i += stride) dst[i] = src[i];
    } else {
        for (uint64_t i = t; i < n; i += stride) dst[i] = src[i];
    }
}

// Streamed result: the consumed lists of events first + i (i < n), contiguous from the first
// one's, into out; the thread of the last event writes the chunk's consumed count to *count.
__global__ void k_fin_cons_chunk(DevPtrs P, uint32_t first, uint32_t n, uint32_t* out, uint32_t* count) {
    const uint32_t base = P.ev_coff[first];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = first + i;
        const uint32_t co = P.ev_coff[e], k = P.rules[P.ev_rule[e]].n_lhs;
        for (uint32_t j = 0; j < k; ++j) out[co - base + j] = P.ev_cons[co + j];
        if (i + 1 == n) *count = co + k - base;
    }
}

// Streamed result: adds the running total tot[w] to the n chunk-local offsets a[0..n).
__global__ void k_fin_rebase(uint32_t* a, uint32_t n, const uint32_t* tot, uint32_t w) {
    const uint32_t base = tot[w];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] += base;
}
// Streamed result: records a chunk's total (sizes[w]) and advances the running total tot[w].
__global__ void k_fin_advance(const uint32_t* chunk_total, uint32_t* tot, uint32_t* sizes, uint32_t w) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sizes[w] = *chunk_total;
        tot[w] += *chunk_total;
    }
}

// ------------------------------------------------------------------------------------------
// Exclusive scan of uint32 (in place allowed), writes the total at out[n]. Three phases:
// per-block sums, one block scans the sums, per-block downsweep.
// ------------------------------------------------------------------------------------------
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanPer = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanPer;

__device__ uint32_t block_excl_scan(uint32_t x, uint32_t* sh, uint32_t& total) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t inc = warp_incl_scan(x);
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        const uint32_t s = lane < (blockDim.x >> 5) ? sh[lane] : 0u;
        const uint32_t si = warp_incl_scan(s);
        sh[lane] = si - s;
        if (lane == 31) sh[32] = si;
    }
    __syncthreads();
    const uint32_t r = sh[w] + inc - x;
    total = sh[32];
    __syncthreads();
    return r;
}

__device__ void k_scan_sums_body(uint32_t* sums, uint32_t nb) {
    __shared__ uint32_t sh[33];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < nb; b += kScanThreads) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t x = i < nb ? sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_excl_scan(x, sh, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}

// Several arrays of the same length scanned by the same launches (blockIdx.y = array).
struct ScanSet {
    const uint32_t* in[4];
    uint32_t* out[4];
};

__global__ void k_scan_reduce(ScanSet S, uint32_t n, uint32_t* sums, uint32_t nb) {
    __shared__ uint32_t sh[33];
    const uint32_t* in = S.in[blockIdx.y];
    const uint32_t base = blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (uint32_t k = 0; k < kScanPer; ++k) {
        const uint32_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0) sums[blockIdx.y * (nb + 1) + blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* sums, uint32_t nb) {
    k_scan_sums_body(sums + blockIdx.x * (nb + 1), nb);
}

// Exclusive scan of one tile per block with the tile carries in `sums` (null: a single tile),
// writing the total at out[n].
__global__ void k_scan_down(ScanSet S, uint32_t n, const uint32_t* sums, uint32_t nb) {
    __shared__ uint32_t sh[33];
    const uint32_t* in = S.in[blockIdx.y];
    uint32_t* out = S.out[blockIdx.y];
    const uint32_t* sm = sums ? sums + blockIdx.y * (nb + 1) : nullptr;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    uint32_t s = 0;
    for (uint32_t k = 0; k < kScanPer; ++k) {
        const uint32_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t ex = block_excl_scan(s, sh, total) + (sm ? sm[blockIdx.x] : 0u);
    for (uint32_t k = 0; k < kScanPer; ++k) {
        const uint32_t i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sm ? sm[nb] : total;
}

}  // namespace hgx
