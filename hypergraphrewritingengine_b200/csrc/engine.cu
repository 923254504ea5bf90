// Host side of the B200 multiway evolution step: device memory, the per-level launch sequence,
// admission of evolutions and result readback. Kernels live in step_kernels.cu (same
// translation unit, so launches need no separate device linking).
#include "engine.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <numeric>

#include "../../include/hgx.h"

#include "step_kernels.cu"

namespace hgx {

namespace {

constexpr int kNumSMs = 148;
constexpr size_t kMaxDynSmem = 227 * 1024;
// Parent regions per warp of the cross-parent lane kernel (measured: 2 beats 4 on C2 and C4).
constexpr uint32_t kLaneRegions = 2;

uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Device-memory ceiling of the engine the calling host thread is driving (HGX_OPT_MAX_DEVICE_BYTES;
// limit 0 = none): the bytes its growable arrays hold, and a growth that would pass the limit
// throws a capacity error before allocating. Set for the duration of every engine call.
struct DeviceBudget {
    uint64_t limit = 0, used = 0;
};
thread_local DeviceBudget* t_budget = nullptr;

struct BudgetScope {
    DeviceBudget* prev;
    explicit BudgetScope(DeviceBudget* b) : prev(t_budget) { t_budget = b; }
    ~BudgetScope() { t_budget = prev; }
};

template <class T>
struct DVec {
    T* p = nullptr;
    size_t cap = 0;
    // Grow to hold n elements, preserving the first `keep`.
    void ensure(size_t n, size_t keep, cudaStream_t s) {
        if (n <= cap) return;
        size_t nc = std::max<size_t>(n, cap + cap / 2 + 1024);
        if (t_budget) {
            const uint64_t add = (nc - cap) * sizeof(T);
            if (t_budget->limit && t_budget->used + add > t_budget->limit)
                throw std::runtime_error("capacity: device memory limit of " +
                                         std::to_string(t_budget->limit) + " bytes reached (the engine "
                                         "holds " + std::to_string(t_budget->used) + " and needs " +
                                         std::to_string(add) + " more)");
            t_budget->used += add;
        }
        T* np = nullptr;
        HGX_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&np), nc * sizeof(T), s));
        if (p && keep) {   // by the SMs, not a copy engine (see k_copy_bytes)
            const uint64_t bytes = std::min(keep, cap) * sizeof(T);
            k_copy_bytes<<<static_cast<uint32_t>(std::min<uint64_t>((bytes + 4095) / 4096, 1184)), 256, 0, s>>>(
                reinterpret_cast<const uint8_t*>(p), reinterpret_cast<uint8_t*>(np), bytes);
            HGX_CUDA_CHECK(cudaGetLastError());
        }
        if (p) HGX_CUDA_CHECK(cudaFreeAsync(p, s));
        p = np;
        cap = nc;
    }
    void release(cudaStream_t s) {
        if (p) cudaFreeAsync(p, s);
        if (t_budget) t_budget->used -= std::min<uint64_t>(t_budget->used, cap * sizeof(T));
        p = nullptr;
        cap = 0;
    }
    size_t bytes() const { return cap * sizeof(T); }
};

// Bytes per element of result array i (the hashes and signatures are u64).
inline uint64_t arr_elem_bytes(int i) {
    if (i == HGX_ARR_STATE_ARITY) return 1;
    return (i == HGX_ARR_STATE_HASH || i == HGX_ARR_EVENT_SIG) ? 8 : 4;
}

struct RuleMax {
    uint32_t rhs = 0, rhs_total = 0, fresh = 0, arity = 1, grow_e = 0, grow_o = 0, stride = 1,
             lhs = 1;
};

DevRule pack_rule(const RuleSpec& r) {
    DevRule d;
    std::memset(&d, 0, sizeof(d));
    if (r.lhs.empty() || r.lhs.size() > kMaxPatternEdges || r.rhs.size() > kMaxPatternEdges)
        throw std::invalid_argument("rule: LHS must have 1..16 edges and RHS at most 16");
    uint32_t lhs_mask = 0, rhs_mask = 0, off = 0;
    d.n_lhs = static_cast<uint8_t>(r.lhs.size());
    d.n_rhs = static_cast<uint8_t>(r.rhs.size());
    for (size_t i = 0; i < r.lhs.size(); ++i) {
        const auto& e = r.lhs[i];
        if (e.empty() || e.size() > kMaxArity) throw std::invalid_argument("rule: LHS edge arity must be 1..16");
        d.lhs_ar[i] = static_cast<uint8_t>(e.size());
        d.lhs_off[i] = static_cast<uint8_t>(off);
        for (uint8_t v : e) {
            if (v >= kMaxVars) throw std::invalid_argument("rule: pattern variable must be < 32");
            if (off >= kMaxSideVars) throw std::invalid_argument("rule: LHS has more than 64 positions");
            d.lhs_vars[off++] = v;
            lhs_mask |= 1u << v;
        }
    }
    d.lhs_total = static_cast<uint8_t>(off);
    off = 0;
    for (size_t i = 0; i < r.rhs.size(); ++i) {
        const auto& e = r.rhs[i];
        if (e.empty() || e.size() > kMaxArity) throw std::invalid_argument("rule: RHS edge arity must be 1..16");
        d.rhs_ar[i] = static_cast<uint8_t>(e.size());
        d.rhs_off[i] = static_cast<uint8_t>(off);
        for (size_t q = 0; q < e.size(); ++q) d.rhs_pos_edge[off + q] = static_cast<uint8_t>(i);
        for (uint8_t v : e) {
            if (v >= kMaxVars) throw std::invalid_argument("rule: pattern variable must be < 32");
            if (off >= kMaxSideVars) throw std::invalid_argument("rule: RHS has more than 64 positions");
            d.rhs_vars[off++] = v;
            rhs_mask |= 1u << v;
        }
    }
    d.rhs_total = static_cast<uint8_t>(off);
    d.new_mask = rhs_mask & ~lhs_mask;
    d.rhs_uni = r.rhs.empty() ? 0 : static_cast<uint8_t>(r.rhs[0].size());
    for (const auto& e : r.rhs)
        if (e.size() != d.rhs_uni) d.rhs_uni = 0;
    {
        // RHS connectivity over its variables (union-find on 32 labels)
        uint8_t up[kMaxVars];
        for (uint32_t v = 0; v < kMaxVars; ++v) up[v] = static_cast<uint8_t>(v);
        auto root = [&](uint32_t x) { while (up[x] != x) x = up[x]; return x; };
        for (const auto& e : r.rhs)
            for (size_t q = 1; q < e.size(); ++q) up[root(e[q])] = static_cast<uint8_t>(root(e[0]));
        uint32_t roots = 0;
        for (uint32_t v = 0; v < kMaxVars; ++v)
            if (((rhs_mask >> v) & 1u) && root(v) == v) ++roots;
        if (roots == 1 && (lhs_mask & ~rhs_mask) == 0) d.flags |= kRuleRhsJoinsLhs;
    }
    uint32_t rank = 0;
    for (uint32_t v = 0; v < kMaxVars; ++v)
        if ((d.new_mask >> v) & 1u) d.fresh_rank[v] = static_cast<uint8_t>(rank++);
    d.n_fresh = static_cast<uint8_t>(rank);
    // Binding schedule: position 0, then the lowest-index position sharing a variable with
    // those already scheduled (else the lowest unscheduled). Fixes the canonical event order.
    std::vector<bool> used(d.n_lhs, false);
    uint32_t bound = 0;
    for (uint32_t s = 0; s < d.n_lhs; ++s) {
        int pick = -1;
        for (uint32_t i = 0; i < d.n_lhs && pick < 0; ++i) {
            if (used[i]) continue;
            uint32_t m = 0;
            for (uint32_t q = 0; q < d.lhs_ar[i]; ++q) m |= 1u << d.lhs_vars[d.lhs_off[i] + q];
            if (s == 0 || (m & bound)) pick = static_cast<int>(i);
        }
        if (pick < 0)
            for (uint32_t i = 0; i < d.n_lhs; ++i)
                if (!used[i]) { pick = static_cast<int>(i); break; }
        used[pick] = true;
        for (uint32_t q = 0; q < d.lhs_ar[pick]; ++q) bound |= 1u << d.lhs_vars[d.lhs_off[pick] + q];
        d.sched[s] = static_cast<uint8_t>(pick);
    }
    return d;
}

uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// A streamed result's level is split into parts of at least this many frontier states.
constexpr uint32_t kStreamPartStates = 16384;
// Results streamed only when the last one was at least this large (a small result's copy is
// shorter than the per-range work streaming adds).
constexpr uint64_t kStreamMinBytes = 64ull << 20;

enum class LayoutKind { Count, Lane, Warp };

// Shared-memory carve-up per warp. Count: the parent and the join. Lane: plus the parent's
// per-vertex occurrence lists and a 32-match batch. Warp: plus the warp-per-child WL arrays.
// NV: the most distinct vertices a staged state of this layout has (0 = bound them by NOCC); the
// warp layout's per-vertex WL arrays and the vertex hash table are sized by it.
Layout make_layout(uint32_t NE, uint32_t NOCC, const RuleMax& rm, LayoutKind kind, bool fwd = false,
                   uint32_t mcap = kLaneJoinCap, bool index = false, uint32_t NV = 0) {
    const bool wl = kind == LayoutKind::Warp;
    const bool lane = kind == LayoutKind::Lane;
    Layout L;
    std::memset(&L, 0, sizeof(L));
    NE = std::max<uint32_t>(NE, 1);
    NOCC = std::max<uint32_t>(NOCC, 1);
    L.NE = NE;
    L.NOCC = NOCC;
    L.CNE = NE + rm.rhs;
    L.CNOCC = NOCC + rm.rhs_total;
    L.NV = NV ? std::min(std::max<uint32_t>(NV, 1), NOCC) : NOCC;
    L.V = L.NV + rm.fresh;
    L.W = (NE + 31) / 32;
    // neighbour-sort entries of one WL round: sum over occurrences of max(a - 1, 1)
    L.NBR = wl ? L.CNOCC * std::max<uint32_t>(rm.arity - 1, 1) : 0;
    uint32_t off = 0;
    auto take = [&](uint32_t bytes, uint32_t align) {
        off = align_up(off, align);
        const uint32_t o = off;
        off += bytes;
        return o;
    };
    if (wl) {
        L.o_cur = take(8 * L.V, 8);
        L.o_nxt = take(8 * L.V, 8);
        L.o_csum = take(8 * L.V, 8);
        L.o_ccnt = take(8 * L.V, 8);
        L.o_nbr = take(8 * L.NBR, 8);
    }
    L.o_peid = take(4 * NE, 4);
    L.o_occ = take(4 * (wl ? L.CNOCC : NOCC), 4);
    L.o_deg = take(4 * (wl ? std::max(L.V, NOCC) : NOCC), 4);   // also load_parent's first-occurrence scratch
    if (wl) {
        L.o_ooff = take(4 * (L.V + 1), 4);
        L.o_nbo = take(4 * (L.V + 1), 4);
        L.o_nn = take(4 * L.V, 4);
        L.o_comp = take(4 * L.V, 4);
    }
    L.o_cand = take(4 * kMaxPatternEdges * L.W, 4);
    L.o_taken = take(4 * L.W, 4);
    L.o_misc = take(4 * kMaxPatternEdges, 4);
    L.o_pevo = take(2 * NE, 2);
    L.o_vloc = take(2 * (NOCC + rm.rhs_total), 2);
    if (wl) L.o_cvo = take(2 * L.CNE, 2);
    L.o_bind = take(2 * kMaxVars, 2);
    L.o_match = take(2 * kMaxPatternEdges, 2);
    L.o_mdepth = take(2 * kMaxPatternEdges, 2);
    L.o_pear = take(NE, 1);
    if (wl) L.o_car = take(L.CNE, 1);
    L.o_rule = take(sizeof(DevRule), 4);
    if (fwd) {
        L.o_fkc = take(4 * kMaxPatternEdges, 4);
        L.o_dkey = take(8 * kFwdCap, 8);
        L.o_dkey2 = take(8 * kFwdCap, 8);
        L.o_fkey = take(8 * 32, 8);
        L.o_dpos = take(2 * kFwdMaxLhs * kFwdCap, 2);
        L.o_dpos2 = take(2 * kFwdMaxLhs * kFwdCap, 2);
        L.o_fpos = take(2 * kFwdMaxLhs * 32, 2);
        L.o_sched2 = take(kMaxPatternEdges, 1);
    }
    if (NOCC > kHashOccMin) {
        L.VT = 64;   // load <= 1/2 over the state's distinct vertices
        while (L.VT < 2 * L.NV) L.VT <<= 1;
        L.o_vtab = take(4 * L.VT, 4);
        L.o_vtid = take(2 * L.VT, 2);
    }
    if (index && !lane && NE > kJoinIndexMin) {
        L.XI = 1;
        L.o_xready = take(4, 4);
        L.o_xoff = take(4 * (NOCC + 1), 4);
        L.o_xinc = take(2 * NOCC, 2);
        L.o_bkey = take(8 * (kSigBuckets + 1), 8);
        L.o_boff = take(4 * (kSigBuckets + 1), 4);
        L.o_blist = take(2 * NE, 2);
    }
    if (wl) {
        uint32_t n2 = 64;   // distinct-colour hash set: >= 2 slots per vertex, + a zero flag
        while (n2 < 2 * L.V) n2 <<= 1;
        L.o_srt = take(8 * (n2 + 1), 8);
    }
    if (lane) {
        L.SB = rm.lhs + rm.rhs_total;
        L.o_poff = take(2 * (kLaneVMax + 1), 2);
        L.o_pocc = take(2 * NOCC, 2);
        L.o_pnoff = take(2 * (kLaneVMax + 1), 2);
        L.o_pnbr = take(2 * NOCC * (rm.arity - 1), 2);
        L.o_pnn = take(2 * kLaneVMax, 2);
        L.o_pconn = take(4, 4);
        L.o_pcnt = take(4 * kLaneVMax, 4);
        L.o_pdeg = take(2 * kLaneVMax, 2);
        L.MCAP = std::max<uint32_t>(1, std::min<uint32_t>(mcap, kLaneJoinCap));
        L.region_bytes = align_up(off, 16);   // batch and match list last: regions >= 1 stop here
        L.o_batch = take(32 * L.SB, 1);
        L.o_mlist = take(4 * L.MCAP, 4);
    }
    L.bytes = align_up(off, 16);
    return L;
}

struct LaunchShape {
    uint32_t grid, block, smem;
};

// Page-locked host memory for results, recycled when a result is freed. Shared with the results
// it hands out, so a result may outlive the engine that produced it. Page-locking is slow (a
// cudaHostAlloc costs far more than the copy it serves), so memory is kept rather than returned:
//   * a result of at most kSmall bytes is carved from a kSlab slab (16-byte aligned, bump
//     pointer); a slab whose results are all freed is reset and reused;
//   * a larger result gets its own power-of-two block; freed blocks are kept (best fit on reuse)
//     up to kKeepBytes in total, the smallest returned to the system beyond that.
struct PinnedPool {
    static constexpr size_t kSmall = 4u << 20, kSlab = 32u << 20;
    static constexpr size_t kKeepBytes = size_t(8) << 30;
    struct Slab {
        uint8_t* base = nullptr;
        size_t top = 0;
        uint32_t live = 0;
    };
    std::mutex mu;
    std::vector<Slab*> slabs;          // every slab (owned)
    Slab* cur = nullptr;               // the slab small results are carved from
    std::vector<std::pair<size_t, void*>> free_blocks;
    size_t free_bytes = 0;

    ~PinnedPool() {
        for (auto& b : free_blocks) cudaFreeHost(b.second);
        for (Slab* sl : slabs) {
            cudaFreeHost(sl->base);
            delete sl;
        }
    }

    // `bytes` of page-locked memory; the returned owner releases it (the pool outlives it).
    static std::shared_ptr<void> acquire(const std::shared_ptr<PinnedPool>& pool, size_t bytes,
                                         uint8_t** out) {
        bytes = std::max<size_t>((bytes + 15) / 16 * 16, 16);
        PinnedPool& P = *pool;
        if (bytes <= kSmall) {
            Slab* sl = nullptr;
            size_t at = 0;
            {
                std::lock_guard<std::mutex> lock(P.mu);
                if (!P.cur || P.cur->top + bytes > kSlab) {
                    P.cur = nullptr;
                    for (Slab* c : P.slabs)
                        if (c->live == 0) { c->top = 0; P.cur = c; break; }
                }
                if (P.cur) {
                    sl = P.cur;
                    at = sl->top;
                    sl->top += bytes;
                    ++sl->live;
                }
            }
            if (!sl) {   // a new slab (allocated outside the lock)
                void* b = nullptr;
                HGX_CUDA_CHECK(cudaHostAlloc(&b, kSlab, cudaHostAllocDefault));
                std::lock_guard<std::mutex> lock(P.mu);
                sl = new Slab;
                sl->base = static_cast<uint8_t*>(b);
                sl->top = bytes;
                sl->live = 1;
                P.slabs.push_back(sl);
                P.cur = sl;
                at = 0;
            }
            *out = sl->base + at;
            return std::shared_ptr<void>(*out, [pool, sl](void*) {
                std::lock_guard<std::mutex> lock(pool->mu);
                --sl->live;
            });
        }
        size_t cap = 0;
        void* p = nullptr;
        {
            std::lock_guard<std::mutex> lock(P.mu);
            size_t best = P.free_blocks.size();
            for (size_t i = 0; i < P.free_blocks.size(); ++i)
                if (P.free_blocks[i].first >= bytes &&
                    (best == P.free_blocks.size() || P.free_blocks[i].first < P.free_blocks[best].first))
                    best = i;
            if (best != P.free_blocks.size()) {
                cap = P.free_blocks[best].first;
                p = P.free_blocks[best].second;
                P.free_bytes -= cap;
                P.free_blocks.erase(P.free_blocks.begin() + best);
            }
        }
        if (!p) {
            size_t pow2 = kSmall * 2;
            while (pow2 < bytes) pow2 <<= 1;
            const size_t step = std::max<size_t>(pow2 / 8, kSmall * 2);   // within 1/8 of the need
            cap = std::max<size_t>((bytes + step - 1) / step * step, kSmall * 2);
            HGX_CUDA_CHECK(cudaHostAlloc(&p, cap, cudaHostAllocDefault));
        }
        *out = static_cast<uint8_t*>(p);
        return std::shared_ptr<void>(p, [pool, cap](void* q) { pool->put(q, cap); });
    }

    void put(void* p, size_t cap) {
        std::lock_guard<std::mutex> lock(mu);
        free_blocks.emplace_back(cap, p);
        free_bytes += cap;
        while (free_bytes > kKeepBytes && !free_blocks.empty()) {   // return the smallest
            auto it = std::min_element(free_blocks.begin(), free_blocks.end());
            free_bytes -= it->first;
            cudaFreeHost(it->second);
            free_blocks.erase(it);
        }
    }
};

}  // namespace

// ==========================================================================================

struct Engine::Impl {
    int device = 0;
    DeviceBudget budget;
    cudaStream_t st = nullptr;
    int timing = 0;   // 0 off, 1 every stage, 2 the expand kernel only
    StageTimes times;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;   // the join autotuner's measurement window
    // Join autotuner for the lane expand kernel: per bucket b = floor(log2(children per frontier
    // state)) and variant (0 warp join, 1 lane walk), the device time per child of large levels
    // (exponential average). Each variant is tried once in the bucket; then the faster one runs
    // (and keeps being measured). Small levels use the measured default (walk from 32
    // children/state).
    struct JoinTuner {
        double ns[8][2] = {};
        uint32_t n[8][2] = {};
    } tuner;
    static constexpr uint64_t kTuneMinChildren = 65536;

    // device arrays
    DVec<DevRule> rules;
    DVec<DevEvo> evos;
    DVec<uint64_t> st_off, st_hash;
    DVec<uint32_t> st_ne, st_nocc, st_evo, st_depth, st_event, st_ev0, st_evn, st_nv, ev_nv;
    DVec<uint32_t> arena;
    DVec<unsigned long long> arena_top;
    DVec<uint32_t> edge_creator;
    DVec<uint32_t> ev_in, ev_rule, ev_coff, ev_prod, ev_fresh, ev_out, ev_cons, ev_cprod;
    DVec<uint8_t> ev_kept;
    DVec<uint64_t> ev_hash;
    DVec<uint32_t> state_of_arrival;
    DVec<unsigned long long> tab_keys;
    DVec<uint32_t> tab_vals;
    DVec<unsigned long long> evo_classes, evo_states, evo_causal;
    DVec<uint32_t> evo_cut, evo_first_ev, evo_last_ev, evo_stopped;
    DVec<uint32_t> err;
    // level temporaries
    DVec<uint32_t> frontier, next_frontier, counts, item_ev, item_cons, item_prod, item_fresh;
    DVec<uint32_t> work, flag_new, scan_new, flag_rep, flag_front, new_state_event, level_max;
    DVec<uint32_t> bcount, boff, bpairs, scan_sums, sync_buf, root_ids;
    DVec<unsigned long long> stats, totals;
    DVec<uint8_t> fmode, fin;
    DVec<uint32_t> fin_cnt, evo_frange, fin_ids, map_s, map_e, frng, slice_off;
    DVec<unsigned long long> evo_new, ev_anc, ev_sig, evo_sigs;
    DVec<unsigned long long> ev_bmask;
    DVec<uint64_t> fin_rng;
    DVec<uint32_t> fin_tab;   // many-evolution finalisation: bases, rule starts, boundary values
    DVec<uint64_t> fin_sec;   // many-evolution finalisation: section offsets
    // Per evolution: the contiguous id ranges it owns, one entry per level (roots first).
    struct EvoRanges {
        std::vector<std::pair<uint32_t, uint32_t>> states, events;
        std::vector<std::pair<uint64_t, uint64_t>> pairs;
        uint32_t roots = 0;
    };
    std::vector<EvoRanges> evo_ranges;
    std::shared_ptr<PinnedPool> pinned = std::make_shared<PinnedPool>();
    uint64_t n_roots_admitted = 0;
    // the per-level read-backs: packed by a kernel straight into mapped page-locked memory (no
    // copy to issue or wait for; the stream's synchronisation makes the writes visible)
    unsigned long long* h_sync = nullptr;
    unsigned long long* d_sync = nullptr;   // h_sync as the device addresses it
    size_t h_sync_words = 0;
    unsigned long long* sync_host(size_t words) {
        if (words > h_sync_words) {
            HGX_CUDA_CHECK(cudaStreamSynchronize(st));
            if (h_sync) HGX_CUDA_CHECK(cudaFreeHost(h_sync));
            h_sync = nullptr;
            const size_t nw = std::max<size_t>(words, 2 * h_sync_words);
            HGX_CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&h_sync), nw * 8, cudaHostAllocMapped));
            HGX_CUDA_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_sync), h_sync, 0));
            h_sync_words = nw;
        }
        return h_sync;
    }

    // Small device-to-host reads and device-to-device copies of the engine stream run on the SMs
    // (k_copy_bytes, into mapped page-locked memory for the reads): they never wait on a copy
    // engine behind the streamed result's copies. sync_st() synchronises the stream and moves the
    // reads to their destinations.
    uint8_t* rb = nullptr;
    size_t rb_cap = 0, rb_top = 0;
    struct RbCopy {
        void* dst;
        size_t off, bytes;
    };
    std::vector<RbCopy> rb_pending;
    static uint32_t copy_grid(uint64_t bytes) {
        return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>((bytes + 4095) / 4096, kNumSMs * 8)));
    }
    void copy_d2d(void* dst, const void* src, uint64_t bytes) {
        if (!bytes) return;
        k_copy_bytes<<<copy_grid(bytes), 256, 0, st>>>(static_cast<const uint8_t*>(src),
                                                       static_cast<uint8_t*>(dst), bytes);
        check_launch();
    }
    void readback(void* dst, const void* src, size_t bytes) {
        if (!bytes) return;
        if (!sr.on) {   // no result copies in flight: a plain copy
            HGX_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
            return;
        }
        const size_t sz = (bytes + 15) / 16 * 16;
        if (rb_top + sz > rb_cap) {
            sync_st();   // the pending reads land first
            if (sz > rb_cap) {
                if (rb) HGX_CUDA_CHECK(cudaFreeHost(rb));
                rb = nullptr;
                rb_cap = std::max<size_t>(sz, std::max<size_t>(2 * rb_cap, 1 << 20));
                HGX_CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&rb), rb_cap, cudaHostAllocMapped));
            }
        }
        uint8_t* d = nullptr;
        HGX_CUDA_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d), rb, 0));
        k_copy_bytes<<<copy_grid(bytes), 256, 0, st>>>(static_cast<const uint8_t*>(src), d + rb_top, bytes);
        check_launch();
        rb_pending.push_back({dst, rb_top, bytes});
        rb_top += sz;
    }
    void sync_st() {
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        for (const RbCopy& c : rb_pending) std::memcpy(c.dst, rb + c.off, c.bytes);
        rb_pending.clear();
        rb_top = 0;
    }

    // ---- streamed result of a single evolution: each finished frontier range's share of the
    // result arrays is finalised on the engine stream into a chunk buffer and copied to the host
    // on the copy stream while the next ranges compute, straight to its final place in the
    // result's per-array page-locked blocks (every array is appended in id order, range by range).
    cudaStream_t cst = nullptr;
    struct ResultStream {
        bool on = false, failed = false, pending = false;
        bool se = false, si = false, causal = false, branchial = false;
        uint32_t R = 0, rule_begin = 0, c0 = 0;
        bool c0_known = false;
        uint64_t s_done = 0, e_done = 0, b_done = 0;      // states / events / pairs streamed
        uint64_t used[ResultArrays::kArrays] = {};        // elements written per array
        uint64_t cap[ResultArrays::kArrays] = {};         // elements of room per array
        uint8_t* h[ResultArrays::kArrays] = {};
        std::shared_ptr<void> own[ResultArrays::kArrays];
        uint64_t tot[4] = {};                             // consumed, causal, state edges, verts
        // the prepared chunk whose copies are not issued yet; every chunk buffer stays allocated
        // until the run's copies are done (a buffer freed on the copy stream and reused on the
        // engine stream would make the engine stream wait for those copies)
        uint8_t* dbuf = nullptr;
        std::vector<uint8_t*> bufs;
        uint64_t doff[ResultArrays::kArrays] = {}, dcount[ResultArrays::kArrays] = {};
        uint32_t* hsz = nullptr;                          // its device-sized counts (page-locked)
        cudaEvent_t ready = nullptr;
    } sr;
    uint64_t sr_hint[ResultArrays::kArrays] = {};        // room the last streamed result needed
    DVec<uint32_t> sr_dev;                               // [0..3] running totals, [4..7] chunk sizes

    // Whether array i's page-locked block has room for `need` elements. Blocks are sized when the
    // stream begins (from the last result of this engine) and never grown: a result that
    // outgrows them is copied whole at the end instead.
    bool sr_room(int i, uint64_t need) {
        if (need <= sr.cap[i]) return true;
        sr.failed = true;
        return false;
    }

    static bool stream_eligible(const RunOptions& opt, size_t nevo) {
        return opt.readback && opt.stream_result && !opt.event_keys && nevo == 1;
    }

    // Streams the result of the (single) evolution just admitted when the engine's last result
    // gives the size of every array (blocks from the pool; small arrays move to small blocks at
    // the end, so a large block goes back to the pool with the run).
    void stream_begin(const RunOptions& opt) {
        sr.on = false;
        if (!stream_eligible(opt, h_evos.size())) return;
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            sr.used[i] = sr.cap[i] = 0;
            sr.h[i] = nullptr;
            sr.own[i].reset();
        }
        uint64_t hinted = 0;
        for (int i = 0; i < ResultArrays::kArrays; ++i) hinted += sr_hint[i] * arr_elem_bytes(i);
        if (!sr_hint[HGX_ARR_STATE_HASH]) return;                           // no result yet
        if (opt.stream_result == 1 && hinted < kStreamMinBytes) return;     // too small to gain
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            if (!sr_hint[i]) continue;
            const uint64_t eb = arr_elem_bytes(i);
            uint8_t* p = nullptr;
            sr.own[i] = PinnedPool::acquire(pinned, sr_hint[i] * eb, &p);
            sr.h[i] = p;
            sr.cap[i] = sr_hint[i];
        }
        for (auto& t : sr.tot) t = 0;
        sr.on = true;
        sr.failed = sr.pending = sr.c0_known = false;
        sr.se = opt.keep_state_edges;
        sr.si = opt.keep_state_edges && opt.keep_state_edge_ids;
        sr.causal = opt.causal;
        sr.branchial = opt.branchial;
        sr.R = static_cast<uint32_t>(n_roots_admitted);
        sr.rule_begin = h_evos[0].rule_begin;
        sr.s_done = 0;
        sr.e_done = sr.R;
        sr.b_done = 0;
        sr_dev.ensure(8, 0, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(sr_dev.p, 0, 8 * sizeof(uint32_t), st));
    }

    // Issues the prepared chunk's copies. The engine stream must have been synchronised since the
    // chunk was prepared (its device-sized counts are then in sr.hsz).
    void stream_issue() {
        if (!sr.pending) return;
        const uint32_t C = sr.hsz[0], K = sr.hsz[1], T = sr.hsz[2], V = sr.hsz[3];
        sr.dcount[HGX_ARR_EVENT_CONS] = C;
        sr.dcount[HGX_ARR_CAUSAL] = 3ull * K;
        sr.dcount[HGX_ARR_STATE_EDGE_IDS] = sr.si ? T : 0;
        sr.dcount[HGX_ARR_STATE_ARITY] = sr.se ? T : 0;
        sr.dcount[HGX_ARR_STATE_VERTS] = sr.se ? V : 0;
        sr.tot[0] += C;
        sr.tot[1] += K;
        sr.tot[2] += T;
        sr.tot[3] += V;
        bool room = true;
        for (int i = 0; i < ResultArrays::kArrays; ++i)
            if (sr.dcount[i]) room = sr_room(i, sr.used[i] + sr.dcount[i] + 1) && room;   // + 1: a closing offset
        if (!room) {
            sr.dbuf = nullptr;
            sr.pending = false;
            return;
        }
        HGX_CUDA_CHECK(cudaStreamWaitEvent(cst, sr.ready, 0));
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            if (!sr.dcount[i]) continue;
            const uint64_t eb = arr_elem_bytes(i);
            HGX_CUDA_CHECK(cudaMemcpyAsync(sr.h[i] + sr.used[i] * eb, sr.dbuf + sr.doff[i],
                                           sr.dcount[i] * eb, cudaMemcpyDeviceToHost, cst));
            sr.used[i] += sr.dcount[i];
        }
        sr.dbuf = nullptr;
        sr.pending = false;
        ++times.result_chunks;
    }

    // After a frontier range: finalise what it added (states [s_done, q3), events [q0, q1), pairs
    // [q4, q5) of the single evolution; q from the range's per-evolution ranges) into a chunk
    // buffer. max_ne / max_no bound the edges and occurrences of its states.
    void stream_prep(const uint32_t* q, uint64_t max_ne, uint64_t max_no) {
        if (!sr.on || sr.failed) return;
        if (sr.pending) {   // no synchronisation since the last chunk: take its counts now
            sync_st();
            stream_issue();
        }
        const uint64_t s1 = std::max<uint64_t>(q[3], sr.s_done);
        const bool ev_any = q[1] > q[0];
        if ((ev_any && q[0] != sr.e_done) || (q[5] > q[4] && q[4] != sr.b_done) ||
            (q[3] > q[2] && q[2] < sr.s_done)) {
            sr.failed = true;   // not one contiguous continuation: the whole result at the end
            return;
        }
        const uint64_t nS = s1 - sr.s_done, nE = ev_any ? q[1] - q[0] : 0;
        const uint64_t nB = (sr.branchial && q[5] > q[4]) ? q[5] - q[4] : 0;
        if (!nS && !nE && !nB) return;
        if (nE && !sr.c0_known) {
            readback(&sr.c0, ev_coff.p + sr.R, 4);
            sync_st();
            sr.c0_known = true;
        }
        const uint64_t Cb = nE * std::max<uint32_t>(rm.lhs, 1);
        const uint64_t Tb = sr.se ? nS * std::max<uint64_t>(max_ne, 1) : 0;
        const uint64_t Vb = sr.se ? nS * std::max<uint64_t>(max_no, 1) : 0;
        // chunk buffer: the result arrays' slices (bounds for the device-sized ones), then the
        // causal counts
        uint64_t cnt[ResultArrays::kArrays] = {nS, nS, 4 * nE, sr.causal ? 3 * Cb : 0, 2 * nB, nE, Cb,
                                               2 * nE, sr.se ? nS + 1 : 0, sr.si ? Tb : 0, Tb,
                                               sr.se ? nS + 1 : 0, Vb, 0};
        uint64_t total = 0;
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            sr.doff[i] = total;
            total += (cnt[i] * arr_elem_bytes(i) + 15) / 16 * 16;
        }
        const uint64_t o_ccnt = total;
        total += (nE + 1) * 4;
        HGX_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&sr.dbuf), std::max<uint64_t>(total, 16), st));
        sr.bufs.push_back(sr.dbuf);
        auto dp = [&](int i) { return reinterpret_cast<uint32_t*>(sr.dbuf + sr.doff[i]); };
        HGX_CUDA_CHECK(cudaMemsetAsync(sr_dev.p + 4, 0, 4 * sizeof(uint32_t), st));
        if (nS) {
            copy_d2d(sr.dbuf + sr.doff[0], st_hash.p + sr.s_done, nS * 8);
            copy_d2d(sr.dbuf + sr.doff[1], st_depth.p + sr.s_done, nS * 4);
        }
        const uint32_t first = static_cast<uint32_t>(q[0]), ne32 = static_cast<uint32_t>(nE);
        if (nE) {
            k_fin_events<<<grid_for(nE, 256), 256, 0, st>>>(ptrs(), first, ne32, sr.rule_begin, dp(2), dp(5),
                                                             dp(7), sr.c0);
            check_launch();
            uint32_t* tmp = sr_dev.p + 4;   // reused: the chunk's consumed count lands in sizes[0]
            k_fin_cons_chunk<<<grid_for(nE, 256), 256, 0, st>>>(ptrs(), first, ne32, dp(6), tmp);
            check_launch();
            k_fin_advance<<<1, 32, 0, st>>>(tmp, sr_dev.p, sr_dev.p + 4, 0);
            check_launch();
            if (sr.causal) {
                uint32_t* ccnt = reinterpret_cast<uint32_t*>(sr.dbuf + o_ccnt);
                k_fin_causal<<<grid_for(nE, 256), 256, 0, st>>>(ptrs(), sr.R, first, ne32, ccnt, nullptr, nullptr, 0);
                check_launch();
                scan(ccnt, ccnt, ne32);
                k_fin_causal<<<grid_for(nE, 256), 256, 0, st>>>(ptrs(), sr.R, first, ne32, nullptr, ccnt, dp(3), 1);
                check_launch();
                k_fin_advance<<<1, 32, 0, st>>>(ccnt + nE, sr_dev.p, sr_dev.p + 4, 1);
                check_launch();
            }
        }
        if (nB) {
            k_fin_shift<<<grid_for(2 * nB, 256), 256, 0, st>>>(bpairs.p + 2 * q[4], 2 * nB, sr.R, dp(4));
            check_launch();
        }
        if (sr.se && nS) {
            const uint32_t s0 = static_cast<uint32_t>(sr.s_done), ns32 = static_cast<uint32_t>(nS);
            scan(st_ne.p + s0, dp(8), ns32);
            scan(st_nocc.p + s0, dp(11), ns32);
            k_fin_states<<<grid_for(nS * 32, 256), 256, 0, st>>>(ptrs(), s0, ns32, dp(8), dp(11),
                                                                sr.si ? dp(9) : nullptr,
                                                                sr.dbuf + sr.doff[10], dp(12));
            check_launch();
            k_fin_rebase<<<grid_for(nS, 256), 256, 0, st>>>(dp(8), ns32, sr_dev.p, 2);
            check_launch();
            k_fin_advance<<<1, 32, 0, st>>>(dp(8) + nS, sr_dev.p, sr_dev.p + 4, 2);
            check_launch();
            k_fin_rebase<<<grid_for(nS, 256), 256, 0, st>>>(dp(11), ns32, sr_dev.p, 3);
            check_launch();
            k_fin_advance<<<1, 32, 0, st>>>(dp(11) + nS, sr_dev.p, sr_dev.p + 4, 3);
            check_launch();
        }
        readback(sr.hsz, sr_dev.p + 4, 4 * sizeof(uint32_t));
        HGX_CUDA_CHECK(cudaEventRecord(sr.ready, st));
        // the element counts known now (the device-sized ones are filled in at issue)
        for (int i = 0; i < ResultArrays::kArrays; ++i) sr.dcount[i] = 0;
        sr.dcount[HGX_ARR_STATE_HASH] = nS;
        sr.dcount[HGX_ARR_STATE_DEPTH] = nS;
        sr.dcount[HGX_ARR_EVENTS] = 4 * nE;
        sr.dcount[HGX_ARR_BRANCHIAL] = 2 * nB;
        sr.dcount[HGX_ARR_EVENT_CONS_OFF] = nE;
        sr.dcount[HGX_ARR_EVENT_PROD] = 2 * nE;
        sr.dcount[HGX_ARR_STATE_EDGE_OFF] = sr.se ? nS : 0;
        sr.dcount[HGX_ARR_STATE_VERT_OFF] = sr.se ? nS : 0;
        sr.pending = true;
        sr.s_done = s1;
        if (nE) sr.e_done = q[1];
        if (q[5] > q[4]) sr.b_done = q[5];
    }

    // Room for the next streamed result: this one's sizes and a sixteenth more.
    void stream_hints(const uint64_t* count) {
        for (int i = 0; i < ResultArrays::kArrays; ++i)
            sr_hint[i] = count[i] ? count[i] + count[i] / 16 + 64 : 0;
        sr_hint[HGX_ARR_STATE_HASH] = std::max<uint64_t>(sr_hint[HGX_ARR_STATE_HASH], 1);
    }

    // The chunk buffers, once the copy stream is done with them.
    void stream_free_bufs() {
        HGX_CUDA_CHECK(cudaStreamSynchronize(cst));
        for (uint8_t* b : sr.bufs) HGX_CUDA_CHECK(cudaFreeAsync(b, st));
        sr.bufs.clear();
    }

    // Drops a stream that could not finish (the result is then finalised whole).
    void stream_abort() {
        sr.dbuf = nullptr;
        sr.pending = false;
        stream_free_bufs();
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            sr.own[i].reset();
            sr.h[i] = nullptr;
            sr.cap[i] = sr.used[i] = 0;
        }
        sr.on = false;
    }

    // The streamed result: the last chunk's copies, the closing offsets, the counts. Empty (no
    // flat arrays) when a block had no room: the caller then finalises the result whole.
    EvolutionResult finalize_streamed() {
        if (sr.s_done < n_states) {   // states no range streamed (the roots of a run of no levels)
            const uint32_t q[7] = {uint32_t(sr.e_done), uint32_t(sr.e_done), uint32_t(sr.s_done),
                                   uint32_t(n_states), uint32_t(sr.b_done), uint32_t(sr.b_done), 0};
            stream_prep(q, ne_bound, nocc_bound);
        }
        if (sr.failed) return {};
        sync_st();
        stream_issue();
        if (sr.failed) return {};
        stream_free_bufs();
        // closing entries of the offset arrays: total consumed / state edges / state vertices
        const int closing[3] = {HGX_ARR_EVENT_CONS_OFF, HGX_ARR_STATE_EDGE_OFF, HGX_ARR_STATE_VERT_OFF};
        const uint64_t value[3] = {sr.tot[0], sr.se ? sr.tot[2] : 0, sr.se ? sr.tot[3] : 0};
        for (int j = 0; j < 3; ++j) {
            const int i = closing[j];
            if (!sr_room(i, sr.used[i] + 1)) break;
            reinterpret_cast<uint32_t*>(sr.h[i])[sr.used[i]] = static_cast<uint32_t>(value[j]);
            sr.used[i] += 1;
        }
        if (sr.failed) return {};
        EvolutionResult r;
        auto owners = std::make_shared<std::vector<std::shared_ptr<void>>>();
        auto flat = std::make_shared<ResultArrays>();
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            const uint64_t eb = arr_elem_bytes(i);
            if (sr.own[i] && sr.used[i] * eb <= PinnedPool::kSmall / 4 &&
                sr.cap[i] * eb > PinnedPool::kSmall) {
                // a small array in a large kept block: move it to a small one, free the large one
                uint8_t* p = nullptr;
                std::shared_ptr<void> own = PinnedPool::acquire(pinned, std::max<uint64_t>(sr.used[i] * eb, 16), &p);
                std::memcpy(p, sr.h[i], sr.used[i] * eb);
                sr.own[i] = std::move(own);
                sr.h[i] = p;
            }
            if (sr.own[i]) owners->push_back(sr.own[i]);
            flat->ptr[i] = sr.h[i];
            flat->count[i] = sr.used[i];
            sr.own[i].reset();
            sr.h[i] = nullptr;
        }
        stream_hints(flat->count);
        flat->owner = owners;
        unsigned long long classes = 0;
        uint32_t stopped = 0;
        readback(&classes, evo_classes.p, 8);
        readback(&stopped, evo_stopped.p, 4);
        sync_st();
        r.flat = flat;
        r.n_roots = sr.R;
        r.num_classes = classes;
        r.n_canonical_events = flat->count[HGX_ARR_EVENT_CONS_OFF] - 1;
        times.result_streamed = 1;
        r.truncated = stopped != 0;
        if (r.truncated)
            r.warnings.push_back(
                "capacity limit reached: the state cap stopped the evolution; the states, events "
                "and relations returned are valid and incomplete");
        sr.on = false;
        return r;
    }

    // host mirrors
    std::vector<DevRule> h_rules;
    std::vector<DevEvo> h_evos;
    std::vector<uint8_t> evo_done, evo_reported;
    std::vector<uint32_t> finished;
    RuleMax rm;
    uint64_t n_states = 0, n_edges = 0, n_events = 0, n_cons = 0, n_bpairs = 0;
    uint64_t next_vertex = 0, arena_words = 0, tab_slots = 0;
    uint32_t frontier_size = 0;
    uint32_t ne_bound = 1, nocc_bound = 1;
    uint64_t launches = 0;

    explicit Impl(int dev) : device(dev) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= dev)
            throw std::runtime_error("hgx: no CUDA device available (the step has no CPU fallback)");
        HGX_CUDA_CHECK(cudaSetDevice(device));
        HGX_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        HGX_CUDA_CHECK(cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking));
        HGX_CUDA_CHECK(cudaEventCreate(&ev_a));
        HGX_CUDA_CHECK(cudaEventCreate(&ev_b));
        HGX_CUDA_CHECK(cudaEventCreateWithFlags(&sr.ready, cudaEventDisableTiming));
        HGX_CUDA_CHECK(cudaMallocHost(reinterpret_cast<void**>(&sr.hsz), 4 * sizeof(uint32_t)));
        cudaMemPool_t pool;
        HGX_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        // (the cross-parent lane kernel also has ~2 KB of static shared memory per block)
        for (const void* k : {(const void*)k_expand_lanes2<false, kLaneRegions>,
                              (const void*)k_expand_lanes2<true, kLaneRegions>,
                              (const void*)k_expand_lanes2<false, kLaneRegions, false>,
                              (const void*)k_expand_lanes2<true, kLaneRegions, false>})
            HGX_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kMaxDynSmem - 8192)));
        for (const void* k : {(const void*)k_count, (const void*)k_expand<true>,
                              (const void*)k_expand<true, true>, (const void*)k_expand<false>,
                              (const void*)k_roots})
            HGX_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kMaxDynSmem)));
        arena_top.ensure(1, 0, st);
        err.ensure(1, 0, st);
        work.ensure(8, 0, st);
        level_max.ensure(8, 0, st);
        sync_buf.ensure(16, 0, st);
        stats.ensure(8, 0, st);
        reset();
    }

    ~Impl() {
        cudaSetDevice(device);
        cudaStreamSynchronize(st);
        for (auto* v : std::initializer_list<DVec<uint32_t>*>{
                 &st_ne, &st_nocc, &st_evo, &st_depth, &st_event, &st_ev0, &st_evn, &st_nv, &ev_nv, &arena,
                 &edge_creator, &ev_in,
                 &ev_rule, &ev_coff, &ev_prod, &ev_fresh, &ev_out, &ev_cons, &ev_cprod,
                 &state_of_arrival, &tab_vals, &evo_cut, &evo_first_ev, &evo_last_ev,
                 &evo_stopped, &err, &frontier, &next_frontier, &counts, &item_ev,
                 &item_cons, &item_prod, &item_fresh, &work, &flag_new, &scan_new, &flag_rep,
                 &flag_front, &new_state_event, &level_max, &bcount, &boff, &bpairs, &scan_sums,
                 &sync_buf, &root_ids})
            v->release(st);
        st_off.release(st);
        st_hash.release(st);
        ev_hash.release(st);
        ev_kept.release(st);
        arena_top.release(st);
        tab_keys.release(st);
        evo_classes.release(st);
        evo_causal.release(st);
        evo_states.release(st);
        stats.release(st);
        totals.release(st);
        fmode.release(st);
        fin.release(st);
        fin_cnt.release(st);
        evo_frange.release(st);
        frng.release(st);
        slice_off.release(st);
        evo_new.release(st);
        ev_anc.release(st);
        ev_bmask.release(st);
        ev_sig.release(st);
        evo_sigs.release(st);
        fin_ids.release(st);
        map_s.release(st);
        map_e.release(st);
        fin_rng.release(st);
        fin_tab.release(st);
        fin_sec.release(st);
        sr_dev.release(st);
        cudaStreamSynchronize(cst);
        for (uint8_t* b : sr.bufs) cudaFreeAsync(b, st);
        cudaStreamDestroy(cst);
        cudaEventDestroy(sr.ready);
        if (sr.hsz) cudaFreeHost(sr.hsz);
        if (rb) cudaFreeHost(rb);
        if (h_sync) cudaFreeHost(h_sync);
        rules.release(st);
        evos.release(st);
        cudaStreamSynchronize(st);
        cudaEventDestroy(ev_a);
        cudaEventDestroy(ev_b);
        for (auto e : ev_pool) cudaEventDestroy(e);
        cudaStreamDestroy(st);
    }

    void reset() {
        if (sr.on) stream_abort();   // a run that ended in an error
        h_rules.clear();
        h_evos.clear();
        evo_ranges.clear();
        evo_done.clear();
        evo_reported.clear();
        finished.clear();
        rm = RuleMax{};
        n_states = n_edges = n_events = n_cons = n_bpairs = 0;
        n_roots_admitted = 0;
        next_vertex = arena_words = tab_slots = 0;
        frontier_size = 0;
        ne_bound = nocc_bound = 1;
        hist = LevelHist{};
        HGX_CUDA_CHECK(cudaMemsetAsync(arena_top.p, 0, sizeof(unsigned long long), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st));
        times = StageTimes{};
        launches = 0;
        pending.clear();
        ev_used = 0;
        HGX_CUDA_CHECK(cudaMemsetAsync(stats.p, 0, 8 * sizeof(unsigned long long), st));
    }

    DevPtrs ptrs() const {
        DevPtrs P;
        P.rules = rules.p;
        P.evos = evos.p;
        P.st_off = st_off.p;
        P.st_ne = st_ne.p;
        P.st_nocc = st_nocc.p;
        P.st_evo = st_evo.p;
        P.st_depth = st_depth.p;
        P.st_event = st_event.p;
        P.st_ev0 = st_ev0.p;
        P.st_evn = st_evn.p;
        P.st_nv = st_nv.p;
        P.ev_nv = ev_nv.p;
        P.st_hash = st_hash.p;
        P.arena = arena.p;
        P.arena_top = arena_top.p;
        P.arena_cap = arena.cap;
        P.edge_creator = edge_creator.p;
        P.ev_in = ev_in.p;
        P.ev_rule = ev_rule.p;
        P.ev_coff = ev_coff.p;
        P.ev_prod = ev_prod.p;
        P.ev_fresh = ev_fresh.p;
        P.ev_out = ev_out.p;
        P.ev_kept = ev_kept.p;
        P.ev_hash = ev_hash.p;
        P.ev_cons = ev_cons.p;
        P.ev_cprod = ev_cprod.p;
        P.ev_anc = ev_anc.p;
        P.ev_bmask = ev_bmask.p;
        P.ev_sig = ev_sig.p;
        P.evo_sigs = evo_sigs.p;
        P.state_of_arrival = state_of_arrival.p;
        P.tab_keys = tab_keys.p;
        P.tab_vals = tab_vals.p;
        P.evo_classes = evo_classes.p;
        P.evo_causal = evo_causal.p;
        P.evo_states = evo_states.p;
        P.evo_cut = evo_cut.p;
        P.evo_first_ev = evo_first_ev.p;
        P.evo_stopped = evo_stopped.p;
        P.err = err.p;
        P.stats = stats.p;
        return P;
    }

    // ---- small helpers ------------------------------------------------------------------
    // Stage timing: CUDA events recorded on the engine stream, no host synchronisation; the
    // pairs are resolved after the run's final synchronise (flush_times).
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    struct Pending { cudaEvent_t a, b; double* acc; };
    std::vector<Pending> pending;
    cudaEvent_t cur_a = nullptr;
    cudaEvent_t next_event() {
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            HGX_CUDA_CHECK(cudaEventCreate(&e));
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }
    void tic(bool expand_kernel = false) {
        if (!(timing == 1 || (timing == 2 && expand_kernel))) return;
        cur_a = next_event();
        HGX_CUDA_CHECK(cudaEventRecord(cur_a, st));
    }
    void toc(double& acc, bool expand_kernel = false) {
        if (!(timing == 1 || (timing == 2 && expand_kernel))) return;
        cudaEvent_t b = next_event();
        HGX_CUDA_CHECK(cudaEventRecord(b, st));
        pending.push_back({cur_a, b, &acc});
    }
    void flush_times() {
        if (pending.empty()) return;
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        for (const auto& p : pending) {
            float ms = 0;
            HGX_CUDA_CHECK(cudaEventElapsedTime(&ms, p.a, p.b));
            *p.acc += ms;
        }
        pending.clear();
        ev_used = 0;
    }
    void check_launch() {
        ++launches;
        HGX_CUDA_CHECK(cudaGetLastError());
    }

    static uint32_t grid_for(uint64_t n, uint32_t block) {
        const uint64_t g = (n + block - 1) / block;
        return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(g, kNumSMs * 16)));
    }

    // Resident blocks per SM of a kernel at a block size and shared-memory size (the driver's
    // occupancy answer, kept: a level asks the same few questions again).
    std::map<std::tuple<const void*, uint32_t, uint32_t>, int> occ_cache;
    int occupancy(const void* kernel, uint32_t block, uint32_t smem) {
        const auto key = std::make_tuple(kernel, block, smem);
        const auto it = occ_cache.find(key);
        if (it != occ_cache.end()) return it->second;
        int bps = 0;
        HGX_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, block, smem));
        bps = std::max(bps, 1);
        occ_cache.emplace(key, bps);
        return bps;
    }

    template <class K>
    LaunchShape warp_shape(K kernel, const Layout& L, uint64_t items) {
        if (L.bytes > kMaxDynSmem)
            throw std::runtime_error("hgx: a state exceeds the per-warp shared-memory capacity (" +
                                     std::to_string(L.bytes) + " bytes needed)");
        uint32_t wpb = static_cast<uint32_t>(std::min<size_t>(8, std::max<size_t>(1, (96 * 1024) / L.bytes)));
        LaunchShape s;
        s.block = 32 * wpb;
        s.smem = L.bytes * wpb;
        int bps = occupancy(reinterpret_cast<const void*>(kernel), s.block, s.smem);
        const uint64_t want = (items + wpb - 1) / wpb;
        s.grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(kNumSMs) * bps)));
        return s;
    }

    // Exclusive scans of k <= 4 arrays of length n (out[n] = total) with the same launches: one
    // launch when n fits one tile, three otherwise.
    void scan_multi(std::initializer_list<std::pair<const uint32_t*, uint32_t*>> arrays, uint32_t n) {
        ScanSet S{};
        uint32_t k = 0;
        for (const auto& a : arrays) { S.in[k] = a.first; S.out[k] = a.second; ++k; }
        const uint32_t nb = (n + kScanTile - 1) / kScanTile;
        if (nb <= 1) {
            k_scan_down<<<dim3(1, k), kScanThreads, 0, st>>>(S, n, nullptr, 0);
            check_launch();
            return;
        }
        scan_sums.ensure(uint64_t(k) * (nb + 1), 0, st);
        k_scan_reduce<<<dim3(nb, k), kScanThreads, 0, st>>>(S, n, scan_sums.p, nb);
        check_launch();
        k_scan_sums<<<k, kScanThreads, 0, st>>>(scan_sums.p, nb);
        check_launch();
        k_scan_down<<<dim3(nb, k), kScanThreads, 0, st>>>(S, n, scan_sums.p, nb);
        check_launch();
    }

    void scan(const uint32_t* in, uint32_t* out, uint32_t n) { scan_multi({{in, out}}, n); }

    // ---- admission ------------------------------------------------------------------------
    //
    // A batch is validated and packed on the host first (nothing changes if a spec is invalid),
    // then uploaded with one copy per array and its roots hashed in one launch.
    uint32_t admit(const EvolutionSpec& spec) { return admit_many({&spec}).front(); }

    std::vector<uint32_t> admit_many(const std::vector<const EvolutionSpec*>& specs) {
        // phase 1: validate and pack (no engine state is touched)
        struct Packed {
            std::vector<DevRule> rules;
            std::vector<uint32_t> words;     // root records with edge ids relative to the batch
            std::vector<uint32_t> nes, noccs;
            std::vector<uint64_t> rel_off;   // record offsets relative to the batch's words
            uint32_t arity = 0;
            uint64_t max_label = 0;
        };
        std::vector<Packed> pk(specs.size());
        uint64_t batch_words = 0, batch_edges = 0;
        for (size_t i = 0; i < specs.size(); ++i) {
            const EvolutionSpec& spec = *specs[i];
            Packed& q = pk[i];
            if (spec.rules.empty()) throw std::invalid_argument("evolve: no rules");
            if (spec.roots.empty()) throw std::invalid_argument("evolve: no initial state");
            for (const auto& r : spec.rules) q.rules.push_back(pack_rule(r));
            for (const auto& root : spec.roots) {
                const uint32_t ne = static_cast<uint32_t>(root.size());
                if (ne == 0) throw std::invalid_argument("evolve: an initial state has no edges");
                uint32_t nocc = 0;
                for (const auto& e : root) {
                    if (e.empty() || e.size() > kMaxArity)
                        throw std::invalid_argument("evolve: initial edge arity must be 1..16");
                    nocc += static_cast<uint32_t>(e.size());
                    q.arity = std::max<uint32_t>(q.arity, static_cast<uint32_t>(e.size()));
                    for (uint32_t v : e) {
                        if (v == kNone) throw std::invalid_argument("evolve: vertex label 4294967295 is reserved");
                        q.max_label = std::max<uint64_t>(q.max_label, v);
                    }
                }
                q.rel_off.push_back(batch_words + q.words.size());
                q.nes.push_back(ne);
                q.noccs.push_back(nocc);
                const uint32_t aw = (ne + 3) / 4;
                const size_t base = q.words.size();
                q.words.resize(base + ne + aw + nocc, 0);
                uint32_t vo = 0;
                for (uint32_t k = 0; k < ne; ++k) {
                    q.words[base + k] = static_cast<uint32_t>(batch_edges + k);   // + n_edges below
                    q.words[base + ne + k / 4] |= static_cast<uint32_t>(root[k].size()) << ((k % 4) * 8);
                    for (uint32_t v : root[k]) q.words[base + ne + aw + vo++] = v;
                }
                batch_edges += ne;
            }
            batch_words += q.words.size();
        }
        if (specs.empty()) return {};

        // phase 2: host mirrors and per-root host arrays
        const uint32_t evo0 = static_cast<uint32_t>(h_evos.size());
        const size_t rules0 = h_rules.size();
        const uint64_t s0 = n_states, a0 = n_events, edges0 = n_edges, arena0 = arena_words, tab0 = tab_slots;
        std::vector<uint32_t> words;
        words.reserve(batch_words);
        std::vector<uint64_t> offs;
        std::vector<uint32_t> nes, noccs, h_evo, h_ev, h_sid, h_front;
        std::vector<uint32_t> ids;
        uint64_t max_label = 0;
        for (size_t i = 0; i < specs.size(); ++i) {
            const EvolutionSpec& spec = *specs[i];
            Packed& q = pk[i];
            const uint32_t evo = evo0 + static_cast<uint32_t>(i);
            DevEvo d;
            std::memset(&d, 0, sizeof(d));
            d.rule_begin = static_cast<uint32_t>(h_rules.size());
            d.rule_count = static_cast<uint32_t>(q.rules.size());
            d.steps = spec.steps;
            d.quotient = spec.quotient ? 1u : 0u;
            d.max_states = spec.max_states;
            for (const DevRule& pr : q.rules) {
                h_rules.push_back(pr);
                rm.rhs = std::max<uint32_t>(rm.rhs, pr.n_rhs);
                rm.rhs_total = std::max<uint32_t>(rm.rhs_total, pr.rhs_total);
                rm.fresh = std::max<uint32_t>(rm.fresh, pr.n_fresh);
                rm.lhs = std::max<uint32_t>(rm.lhs, pr.n_lhs);
                for (uint32_t k = 0; k < pr.n_rhs; ++k) rm.arity = std::max<uint32_t>(rm.arity, pr.rhs_ar[k]);
                rm.grow_e = std::max<int>(rm.grow_e, int(pr.n_rhs) - int(pr.n_lhs));
                rm.grow_o = std::max<int>(rm.grow_o, int(pr.rhs_total) - int(pr.lhs_total));
            }
            rm.stride = std::max<uint32_t>(rm.stride, d.rule_count);
            rm.arity = std::max<uint32_t>(rm.arity, q.arity);
            max_label = std::max(max_label, q.max_label);
            const uint32_t nr = static_cast<uint32_t>(q.nes.size());
            for (uint32_t k = 0; k < nr; ++k) {
                const uint32_t ne = q.nes[k];
                ne_bound = std::max(ne_bound, ne);
                nocc_bound = std::max(nocc_bound, q.noccs[k]);
                offs.push_back(arena0 + q.rel_off[k]);
                nes.push_back(ne);
                noccs.push_back(q.noccs[k]);
                const uint32_t sid = static_cast<uint32_t>(s0 + h_sid.size());
                h_ev.push_back(static_cast<uint32_t>(a0 + h_sid.size()));
                h_sid.push_back(sid);
                h_evo.push_back(evo);
                if (spec.steps > 0) h_front.push_back(sid);
            }
            // edge ids in the records are relative to the batch: shift by the edge counter
            {
                size_t base = 0;
                for (uint32_t k = 0; k < nr; ++k) {
                    const uint32_t ne = q.nes[k], aw = (ne + 3) / 4;
                    for (uint32_t j = 0; j < ne; ++j) q.words[base + j] += static_cast<uint32_t>(edges0);
                    base += ne + aw + q.noccs[k];
                }
            }
            words.insert(words.end(), q.words.begin(), q.words.end());
            // dedup table region
            const uint64_t cap = next_pow2(std::max<uint64_t>(256, 4ull * nr));
            d.table_off = tab_slots;
            d.table_mask = cap - 1;
            tab_slots += cap + 1;
            evo_ranges.emplace_back();
            evo_ranges.back().states.emplace_back(static_cast<uint32_t>(s0 + h_sid.size() - nr),
                                                  static_cast<uint32_t>(s0 + h_sid.size()));
            evo_ranges.back().roots = nr;
            h_evos.push_back(d);
            evo_done.push_back(spec.steps > 0 ? 0 : 1);
            evo_reported.push_back(0);
            if (spec.steps == 0) finished.push_back(evo);
            ids.push_back(evo);
        }
        const uint32_t nr = static_cast<uint32_t>(h_sid.size());
        const size_t nevo = h_evos.size(), nnew = nevo - evo0;
        n_edges += batch_edges;
        next_vertex = std::max<uint64_t>(next_vertex, max_label + 1);

        // phase 3: device arrays, one copy or fill per array
        auto up = [&](auto* dst, const auto& src) {
            if (!src.empty())
                HGX_CUDA_CHECK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(src[0]), cudaMemcpyHostToDevice, st));
        };
        tab_keys.ensure(tab_slots, tab0, st);
        tab_vals.ensure(tab_slots, tab0, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(tab_keys.p + tab0, 0, (tab_slots - tab0) * sizeof(unsigned long long), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(tab_vals.p + tab0, 0xFF, (tab_slots - tab0) * sizeof(uint32_t), st));
        rules.ensure(h_rules.size(), rules0, st);
        HGX_CUDA_CHECK(cudaMemcpyAsync(rules.p + rules0, h_rules.data() + rules0,
                                       (h_rules.size() - rules0) * sizeof(DevRule), cudaMemcpyHostToDevice, st));
        evos.ensure(nevo, evo0, st);
        HGX_CUDA_CHECK(cudaMemcpyAsync(evos.p + evo0, &h_evos[evo0], nnew * sizeof(DevEvo), cudaMemcpyHostToDevice, st));
        evo_classes.ensure(nevo, evo0, st);
        evo_causal.ensure(nevo, evo0, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_causal.p + evo0, 0, nnew * sizeof(unsigned long long), st));
        evo_states.ensure(nevo, evo0, st);
        evo_sigs.ensure(nevo, evo0, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_sigs.p + evo0, 0, nnew * sizeof(unsigned long long), st));
        evo_cut.ensure(nevo, evo0, st);
        evo_first_ev.ensure(nevo, evo0, st);
        evo_last_ev.ensure(nevo, evo0, st);
        evo_stopped.ensure(nevo, evo0, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_classes.p + evo0, 0, nnew * sizeof(unsigned long long), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_states.p + evo0, 0, nnew * sizeof(unsigned long long), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_cut.p + evo0, 0xFF, nnew * sizeof(uint32_t), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_stopped.p + evo0, 0, nnew * sizeof(uint32_t), st));
        arena.ensure(arena0 + words.size(), arena0, st);
        up(arena.p + arena0, words);
        arena_words += words.size();
        const unsigned long long top = arena_words;
        HGX_CUDA_CHECK(cudaMemcpyAsync(arena_top.p, &top, sizeof(top), cudaMemcpyHostToDevice, st));
        edge_creator.ensure(n_edges, edges0, st);   // initial edges have no producer
        HGX_CUDA_CHECK(cudaMemsetAsync(edge_creator.p + edges0, 0xFF, batch_edges * sizeof(uint32_t), st));
        grow_states(s0 + nr);
        grow_events(a0 + nr);
        std::vector<uint32_t> h_zero(nr, 0), h_none(nr, kNone);
        std::vector<uint8_t> h_kept(nr, 0);
        up(st_off.p + s0, offs);
        up(st_ne.p + s0, nes);
        up(st_nocc.p + s0, noccs);
        up(st_evo.p + s0, h_evo);
        up(st_depth.p + s0, h_zero);
        up(st_event.p + s0, h_ev);
        up(ev_in.p + a0, h_none);
        up(ev_out.p + a0, h_sid);
        up(ev_kept.p + a0, h_kept);
        up(state_of_arrival.p + a0, h_sid);
        n_states += nr;
        n_events += nr;
        n_roots_admitted += nr;

        // hash the roots on the device and seed the tables
        root_ids.ensure(nr, 0, st);
        up(root_ids.p, h_sid);
        RuleMax none;
        none.arity = rm.arity;
        const uint32_t mne = *std::max_element(nes.begin(), nes.end());
        const uint32_t mno = *std::max_element(noccs.begin(), noccs.end());
        Layout L = make_layout(mne, mno, none, LayoutKind::Warp);
        HGX_CUDA_CHECK(cudaMemsetAsync(work.p, 0, 8 * sizeof(uint32_t), st));
        LaunchShape sh = warp_shape(k_roots, L, nr);
        tic();
        k_roots<<<sh.grid, sh.block, sh.smem, st>>>(ptrs(), root_ids.p, nr, work.p, L);
        check_launch();
        hist.have_ok = false;   // the roots move the class and state counters
        k_root_counts<<<grid_for(nr, 256), 256, 0, st>>>(ptrs(), root_ids.p, nr);
        check_launch();
        toc(times.roots);

        if (!h_front.empty()) {
            frontier.ensure(frontier_size + h_front.size(), frontier_size, st);
            up(frontier.p + frontier_size, h_front);
            frontier_size += static_cast<uint32_t>(h_front.size());
        }
        return ids;
    }

    void grow_states(uint64_t n) {
        const uint64_t k = n_states;
        st_off.ensure(n, k, st);
        st_hash.ensure(n, k, st);
        st_ne.ensure(n, k, st);
        st_nocc.ensure(n, k, st);
        st_evo.ensure(n, k, st);
        st_depth.ensure(n, k, st);
        st_event.ensure(n, k, st);
        st_ev0.ensure(n, k, st);
        st_evn.ensure(n, k, st);
        st_nv.ensure(n, k, st);
    }

    void grow_events(uint64_t n) {
        const uint64_t k = n_events;
        ev_in.ensure(n, k, st);
        ev_rule.ensure(n, k, st);
        ev_coff.ensure(n, k, st);
        ev_prod.ensure(n, k, st);
        ev_fresh.ensure(n, k, st);
        ev_out.ensure(n, k, st);
        ev_kept.ensure(n, k, st);
        ev_hash.ensure(n, k, st);
        ev_nv.ensure(n, k, st);
        state_of_arrival.ensure(n, k, st);
    }

    // Rebuild an evolution's dedup table at a larger capacity.
    // A new, larger table region for (off, mask) holding `need` keys at load <= 1/2; the old
    // region (if any, mask != 0) is rehashed into it. The caller uploads the changed h_evos.
    void regrow_region(uint64_t& off, uint64_t& mask, uint64_t need) {
        const uint64_t cap = next_pow2(std::max<uint64_t>({need * 2, mask ? (mask + 1) * 2 : 0, 256}));
        const uint64_t noff = tab_slots;
        const uint64_t new_slots = tab_slots + cap + 1;
        tab_keys.ensure(new_slots, tab_slots, st);
        tab_vals.ensure(new_slots, tab_slots, st);
        HGX_CUDA_CHECK(cudaMemsetAsync(tab_keys.p + noff, 0, (cap + 1) * sizeof(unsigned long long), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(tab_vals.p + noff, 0xFF, (cap + 1) * sizeof(uint32_t), st));
        tab_slots = new_slots;
        if (mask) {
            k_rehash<<<grid_for(mask + 2, 256), 256, 0, st>>>(tab_keys.p, tab_vals.p, off, mask, noff,
                                                             cap - 1, err.p);
            check_launch();
        }
        off = noff;
        mask = cap - 1;
    }

    void regrow_table(uint32_t evo, uint64_t need) {
        regrow_region(h_evos[evo].table_off, h_evos[evo].table_mask, need);
    }

    // Upload h_evos[lo, hi) (one copy for all the tables a level regrew).
    void upload_evos(size_t lo, size_t hi) {
        if (hi > lo)
            HGX_CUDA_CHECK(cudaMemcpyAsync(evos.p + lo, &h_evos[lo], (hi - lo) * sizeof(DevEvo),
                                           cudaMemcpyHostToDevice, st));
    }



    // Single-evolution result, finalised on the device and copied to a pinned block at once.
    EvolutionResult finalize_single(const RunOptions& opt) {
        EvolutionResult r;
        const uint32_t R = static_cast<uint32_t>(n_roots_admitted);
        uint32_t cut = kNone, stopped = 0;
        unsigned long long classes = 0;
        HGX_CUDA_CHECK(cudaMemcpyAsync(&cut, evo_cut.p, 4, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(&stopped, evo_stopped.p, 4, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(&classes, evo_classes.p, 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        const uint64_t e_end = stopped ? std::min<uint64_t>(n_events, cut) : n_events;
        const uint32_t E = static_cast<uint32_t>(e_end - R);
        const uint32_t S = static_cast<uint32_t>(n_states);
        const uint64_t B = opt.branchial ? n_bpairs : 0;
        // consumed lists of the kept events are one contiguous range [c0, c0 + C)
        uint32_t c0 = 0, clast = 0, rlast = 0;
        if (E) {
            HGX_CUDA_CHECK(cudaMemcpyAsync(&c0, ev_coff.p + R, 4, cudaMemcpyDeviceToHost, st));
            HGX_CUDA_CHECK(cudaMemcpyAsync(&clast, ev_coff.p + e_end - 1, 4, cudaMemcpyDeviceToHost, st));
            HGX_CUDA_CHECK(cudaMemcpyAsync(&rlast, ev_rule.p + e_end - 1, 4, cudaMemcpyDeviceToHost, st));
        }
        // causal counts and state CSR offsets
        fin_cnt.ensure(uint64_t(E) + 1 + 2ull * (S + 1), 0, st);
        uint32_t* ccnt = fin_cnt.p;                 // [E+1] counts, then scanned in place
        uint32_t* eoff = fin_cnt.p + E + 1;         // [S+1]
        uint32_t* voff = eoff + S + 1;              // [S+1]
        if (E && opt.causal) {
            k_fin_causal<<<grid_for(E, 256), 256, 0, st>>>(ptrs(), R, R, E, ccnt, nullptr, nullptr, 0);
            check_launch();
            scan(ccnt, ccnt, E);
        } else {
            HGX_CUDA_CHECK(cudaMemsetAsync(ccnt + E, 0, 4, st));
        }
        if (opt.keep_state_edges) {
            scan(st_ne.p, eoff, S);
            scan(st_nocc.p, voff, S);
        }
        uint32_t K = 0, T = 0, V = 0;
        HGX_CUDA_CHECK(cudaMemcpyAsync(&K, ccnt + E, 4, cudaMemcpyDeviceToHost, st));
        if (opt.keep_state_edges) {
            HGX_CUDA_CHECK(cudaMemcpyAsync(&T, eoff + S, 4, cudaMemcpyDeviceToHost, st));
            HGX_CUDA_CHECK(cudaMemcpyAsync(&V, voff + S, 4, cudaMemcpyDeviceToHost, st));
        }
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        const uint32_t C = E ? clast + h_rules[rlast].n_lhs - c0 : 0;
        const bool se = opt.keep_state_edges;
        const bool si = se && opt.keep_state_edge_ids;
        // host block layout (hgx_array order), 16-byte aligned sections
        const bool sg = opt.event_keys != 0;
        uint64_t count[ResultArrays::kArrays] = {
            S, S, 4ull * E, 3ull * K, 2 * B, uint64_t(E) + 1, C, 2ull * E,
            se ? S + 1ull : 1, si ? T : 0, se ? T : 0, se ? S + 1ull : 1, se ? V : 0, sg ? E : 0};
        uint64_t off[ResultArrays::kArrays];
        uint64_t total = 0;
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            off[i] = total;
            total += (count[i] * arr_elem_bytes(i) + 15) / 16 * 16;
        }
        // device staging for the derived arrays (same layout; direct arrays are copied from
        // their own device buffers)
        fin.ensure(total, 0, st);
        uint8_t* d = fin.p;
        auto dp = [&](int i) { return reinterpret_cast<uint32_t*>(d + off[i]); };
        if (E) {
            k_fin_events<<<grid_for(E, 256), 256, 0, st>>>(ptrs(), R, E, h_evos[0].rule_begin, dp(2),
                                                             dp(5), dp(7), c0);
            check_launch();
            HGX_CUDA_CHECK(cudaMemcpyAsync(dp(5) + E, &C, 4, cudaMemcpyHostToDevice, st));
        } else {
            HGX_CUDA_CHECK(cudaMemsetAsync(dp(5), 0, 4, st));
        }
        if (K) {
            k_fin_causal<<<grid_for(E, 256), 256, 0, st>>>(ptrs(), R, R, E, nullptr, ccnt, dp(3), 1);
            check_launch();
        }
        if (B) {
            k_fin_shift<<<grid_for(2 * B, 256), 256, 0, st>>>(bpairs.p, 2 * B, R, dp(4));
            check_launch();
        }
        if (se) {
            k_fin_states<<<grid_for(uint64_t(S) * 32, 256), 256, 0, st>>>(ptrs(), 0, S, eoff, voff,
                                                                         si ? dp(9) : nullptr,
                                                                         d + off[10], dp(12));
            check_launch();
        } else {
            HGX_CUDA_CHECK(cudaMemsetAsync(dp(8), 0, 4, st));
            HGX_CUDA_CHECK(cudaMemsetAsync(dp(11), 0, 4, st));
        }
        uint8_t* h = nullptr;
        auto flat = std::make_shared<ResultArrays>();
        flat->owner = PinnedPool::acquire(pinned, total, &h);
        auto d2h_from = [&](int i, const void* src) {
            const size_t bytes = count[i] * arr_elem_bytes(i);
            if (bytes) HGX_CUDA_CHECK(cudaMemcpyAsync(h + off[i], src, bytes, cudaMemcpyDeviceToHost, st));
        };
        d2h_from(0, st_hash.p);
        d2h_from(1, st_depth.p);
        d2h_from(6, ev_cons.p + c0);
        if (sg) d2h_from(HGX_ARR_EVENT_SIG, ev_sig.p + R);
        if (se) {
            d2h_from(8, eoff);
            d2h_from(11, voff);
        }
        // the derived sections, in one copy from the first through the last derived array
        for (int i : {2, 3, 4, 5, 7}) d2h_from(i, d + off[i]);
        if (se) for (int i : {9, 10, 12}) d2h_from(i, d + off[i]);
        if (!se) {
            std::memset(h + off[8], 0, 4);
            std::memset(h + off[11], 0, 4);
        }
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        for (int i = 0; i < ResultArrays::kArrays; ++i) {
            flat->ptr[i] = h + off[i];
            flat->count[i] = count[i];
        }
        r.flat = flat;
        r.n_roots = R;
        r.num_classes = classes;
        r.n_canonical_events = E;
        if (sg) {
            unsigned long long nsig = 0;
            HGX_CUDA_CHECK(cudaMemcpyAsync(&nsig, evo_sigs.p, 8, cudaMemcpyDeviceToHost, st));
            HGX_CUDA_CHECK(cudaStreamSynchronize(st));
            r.n_canonical_events = nsig;
        }
        r.truncated = stopped != 0;
        if (r.truncated)
            r.warnings.push_back(
                "capacity limit reached: the state cap stopped the evolution; the states, events "
                "and relations returned are valid and incomplete");
        return r;
    }


    // Many evolutions finalised on the device at once, from their recorded id ranges: one set of
    // launches, one staging block, one copy into one page-locked block that every result shares.
    std::vector<EvolutionResult> finalize_many(const std::vector<uint32_t>& which, const RunOptions& opt) {
        const uint32_t K = static_cast<uint32_t>(which.size());
        std::vector<EvolutionResult> out(K);
        if (!K) return out;
        const bool se = opt.keep_state_edges, sg = opt.event_keys != 0;
        const bool si = se && opt.keep_state_edge_ids;
        // concatenated id ranges (states, events, pairs) and each evolution's start in them
        std::vector<uint64_t> rs, rc, re, rce, rp, rcp;
        std::vector<uint32_t> tab(4 * (K + 1) + K, 0);
        uint32_t* sb = tab.data();
        uint32_t* eb = sb + (K + 1);
        uint32_t* pb = eb + (K + 1);
        uint32_t* rb = pb + (K + 1);
        uint64_t S = 0, E = 0, B = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const EvoRanges& er = evo_ranges.at(which[k]);
            sb[k] = static_cast<uint32_t>(S);
            eb[k] = static_cast<uint32_t>(E);
            pb[k] = static_cast<uint32_t>(B);
            rb[k] = h_evos[which[k]].rule_begin;
            for (auto& q : er.states) { rs.push_back(q.first); rc.push_back(S); S += q.second - q.first; }
            for (auto& q : er.events) { re.push_back(q.first); rce.push_back(E); E += q.second - q.first; }
            if (opt.branchial)
                for (auto& q : er.pairs) { rp.push_back(q.first); rcp.push_back(B); B += q.second - q.first; }
        }
        if (S + E >= 0xFFFFFFF0ull || B >= 0xFFFFFFF0ull)
            throw std::runtime_error("hgx: result too large for one finalisation");
        sb[K] = static_cast<uint32_t>(S);
        eb[K] = static_cast<uint32_t>(E);
        pb[K] = static_cast<uint32_t>(B);
        const uint32_t NS = static_cast<uint32_t>(S), NE = static_cast<uint32_t>(E);
        // device tables: ranges (u64) and bases (u32)
        std::vector<uint64_t> rng;
        const uint64_t o_rs = 0, o_rc = rs.size(), o_re = 2 * rs.size(), o_rce = o_re + re.size(),
                       o_rp = o_rce + re.size(), o_rcp = o_rp + rp.size();
        rng.reserve(o_rcp + rp.size());
        for (auto* v : {&rs, &rc, &re, &rce, &rp, &rcp}) rng.insert(rng.end(), v->begin(), v->end());
        fin_rng.ensure(std::max<size_t>(rng.size(), 1), 0, st);
        HGX_CUDA_CHECK(cudaMemcpyAsync(fin_rng.p, rng.data(), rng.size() * 8, cudaMemcpyHostToDevice, st));
        fin_tab.ensure(tab.size() + 4 * (K + 1), 0, st);
        HGX_CUDA_CHECK(cudaMemcpyAsync(fin_tab.p, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, st));
        const uint32_t* d_sb = fin_tab.p;
        const uint32_t* d_eb = d_sb + (K + 1);
        const uint32_t* d_pb = d_eb + (K + 1);
        const uint32_t* d_rb = d_pb + (K + 1);
        uint32_t* d_bounds = fin_tab.p + tab.size();
        // ids, global -> local maps
        fin_ids.ensure(S + E + 1, 0, st);
        uint32_t* sids = fin_ids.p;
        uint32_t* eids = fin_ids.p + S;
        k_expand_ranges<<<grid_for(S, 256), 256, 0, st>>>(fin_rng.p + o_rs, fin_rng.p + o_rc,
                                                          static_cast<uint32_t>(rs.size()), S, sids);
        check_launch();
        if (E) {
            k_expand_ranges<<<grid_for(E, 256), 256, 0, st>>>(fin_rng.p + o_re, fin_rng.p + o_rce,
                                                              static_cast<uint32_t>(re.size()), E, eids);
            check_launch();
        }
        map_s.ensure(n_states, 0, st);
        map_e.ensure(n_events, 0, st);
        k_map_multi<<<grid_for(S, 256), 256, 0, st>>>(sids, NS, d_sb, K, map_s.p);
        check_launch();
        if (E) {
            k_map_multi<<<grid_for(E, 256), 256, 0, st>>>(eids, NE, d_eb, K, map_e.p);
            check_launch();
        }
        // sizes and their scans: state edges / occurrences, event consumed / causal entries
        fin_cnt.ensure(2ull * (S + 1) + 2ull * (E + 1), 0, st);
        uint32_t* sne = fin_cnt.p;
        uint32_t* sno = sne + S + 1;
        uint32_t* ecc = sno + S + 1;
        uint32_t* ekc = ecc + E + 1;
        k_fin_states_multi<<<grid_for(S, 256), 256, 0, st>>>(ptrs(), sids, NS, d_sb, K, nullptr, nullptr, sne, sno);
        check_launch();
        scan(sne, sne, NS);
        scan(sno, sno, NS);
        if (E) {
            k_fin_events_multi<<<grid_for(E, 256), 256, 0, st>>>(ptrs(), eids, NE, d_eb, K, d_rb, map_s.p, map_e.p,
                                                                 ecc, ekc, nullptr, nullptr, nullptr, nullptr,
                                                                 0, opt.causal ? 1 : 0, 0);
            check_launch();
        }
        scan(ecc, ecc, NE);
        scan(ekc, ekc, NE);
        k_fin_bounds<<<grid_for(K + 1, 256), 256, 0, st>>>(sne, d_sb, K, d_bounds);
        k_fin_bounds<<<grid_for(K + 1, 256), 256, 0, st>>>(sno, d_sb, K, d_bounds + (K + 1));
        k_fin_bounds<<<grid_for(K + 1, 256), 256, 0, st>>>(ecc, d_eb, K, d_bounds + 2 * (K + 1));
        k_fin_bounds<<<grid_for(K + 1, 256), 256, 0, st>>>(ekc, d_eb, K, d_bounds + 3 * (K + 1));
        check_launch();
        std::vector<uint32_t> bnd(4 * (K + 1));
        const size_t nevo = h_evos.size();
        std::vector<unsigned long long> cls(nevo), sigs(nevo, 0);
        std::vector<uint32_t> stop(nevo);
        HGX_CUDA_CHECK(cudaMemcpyAsync(bnd.data(), d_bounds, bnd.size() * 4, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(cls.data(), evo_classes.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(stop.data(), evo_stopped.p, nevo * 4, cudaMemcpyDeviceToHost, st));
        if (sg) HGX_CUDA_CHECK(cudaMemcpyAsync(sigs.data(), evo_sigs.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        // sections: each evolution's arrays, in hgx_array order, 16-byte aligned
        std::vector<uint64_t> sec(uint64_t(K) * kArr), cnt(uint64_t(K) * kArr);
        uint64_t total = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const uint64_t Sk = sb[k + 1] - sb[k], Ek = eb[k + 1] - eb[k], Bk = pb[k + 1] - pb[k];
            const uint64_t Tk = bnd[k + 1] - bnd[k], Vk = bnd[K + 1 + k + 1] - bnd[K + 1 + k];
            const uint64_t Ck = bnd[2 * (K + 1) + k + 1] - bnd[2 * (K + 1) + k];
            const uint64_t Kk = bnd[3 * (K + 1) + k + 1] - bnd[3 * (K + 1) + k];
            const uint64_t c[kArr] = {Sk, Sk, 4 * Ek, 3 * Kk, 2 * Bk, Ek + 1, Ck, 2 * Ek,
                                      se ? Sk + 1 : 1, si ? Tk : 0, se ? Tk : 0, se ? Sk + 1 : 1,
                                      se ? Vk : 0, sg ? Ek : 0};
            for (uint32_t a = 0; a < kArr; ++a) {
                sec[uint64_t(k) * kArr + a] = total;
                cnt[uint64_t(k) * kArr + a] = c[a];
                total += (c[a] * arr_elem_bytes(static_cast<int>(a)) + 15) / 16 * 16;
            }
        }
        fin.ensure(std::max<uint64_t>(total, 16), 0, st);
        fin_sec.ensure(sec.size(), 0, st);
        HGX_CUDA_CHECK(cudaMemcpyAsync(fin_sec.p, sec.data(), sec.size() * 8, cudaMemcpyHostToDevice, st));
        uint8_t* stage = fin.p;
        const uint64_t* d_sec = fin_sec.p;
        // emit
        k_fin_states_multi<<<grid_for(S, 256), 256, 0, st>>>(ptrs(), sids, NS, d_sb, K, stage, d_sec, nullptr, nullptr);
        check_launch();
        if (se) {
            k_fin_offsets_multi<<<grid_for(S + K, 256), 256, 0, st>>>(sne, NS, d_sb, K, stage, d_sec, HGX_ARR_STATE_EDGE_OFF);
            k_fin_offsets_multi<<<grid_for(S + K, 256), 256, 0, st>>>(sno, NS, d_sb, K, stage, d_sec, HGX_ARR_STATE_VERT_OFF);
            check_launch();
            k_fin_records_multi<<<grid_for(S * 32, 256), 256, 0, st>>>(ptrs(), sids, NS, d_sb, K, sne, sno, stage, d_sec,
                                                                        si ? 1 : 0);
            check_launch();
        } else {
            k_fin_zero_multi<<<grid_for(K, 256), 256, 0, st>>>(stage, d_sec, K, HGX_ARR_STATE_EDGE_OFF);
            k_fin_zero_multi<<<grid_for(K, 256), 256, 0, st>>>(stage, d_sec, K, HGX_ARR_STATE_VERT_OFF);
            check_launch();
        }
        k_fin_offsets_multi<<<grid_for(E + K, 256), 256, 0, st>>>(ecc, NE, d_eb, K, stage, d_sec, HGX_ARR_EVENT_CONS_OFF);
        check_launch();
        if (E) {
            k_fin_events_multi<<<grid_for(E, 256), 256, 0, st>>>(ptrs(), eids, NE, d_eb, K, d_rb, map_s.p, map_e.p,
                                                                 nullptr, nullptr, ecc, ekc, stage, d_sec,
                                                                 1, opt.causal ? 1 : 0, sg ? 1 : 0);
            check_launch();
        }
        if (B) {
            k_fin_pairs_multi<<<grid_for(B, 256), 256, 0, st>>>(bpairs.p, fin_rng.p + o_rp, fin_rng.p + o_rcp,
                                                                static_cast<uint32_t>(rp.size()), B, d_pb, K,
                                                                map_e.p, stage, d_sec);
            check_launch();
        }
        uint8_t* h = nullptr;
        std::shared_ptr<void> owner = PinnedPool::acquire(pinned, std::max<uint64_t>(total, 16), &h);
        if (total) HGX_CUDA_CHECK(cudaMemcpyAsync(h, stage, total, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        for (uint32_t k = 0; k < K; ++k) {
            const uint32_t evo = which[k];
            auto flat = std::make_shared<ResultArrays>();
            flat->owner = owner;
            for (uint32_t a = 0; a < kArr; ++a) {
                flat->ptr[a] = h + sec[uint64_t(k) * kArr + a];
                flat->count[a] = cnt[uint64_t(k) * kArr + a];
            }
            EvolutionResult& r = out[k];
            r.flat = flat;
            r.n_roots = evo_ranges[evo].roots;
            r.num_classes = cls[evo];
            r.truncated = stop[evo] != 0;
            r.n_canonical_events = sg ? sigs[evo] : (eb[k + 1] - eb[k]);
            if (r.truncated)
                r.warnings.push_back(
                    "capacity limit reached: the state cap stopped the evolution; the states, events "
                    "and relations returned are valid and incomplete");
        }
        return out;
    }


    // Causal triples are written even when the caller did not ask for them; they then land in
    // this scratch instead of the result.

    // Counts only (results stay on the device): events and branchial pairs from the recorded
    // per-evolution ranges; states, classes and causal triples from the device counters (the
    // causal ones counted level by level in k_outstate).
    void read_counts(const std::vector<uint32_t>& which, std::vector<EvolutionResult>& out,
                     bool signatures) {
        const size_t nevo = h_evos.size();
        std::vector<unsigned long long> causal(nevo), cls(nevo), sts(nevo), sig(nevo, 0);
        std::vector<uint32_t> stop(nevo);
        if (signatures)
            HGX_CUDA_CHECK(cudaMemcpyAsync(sig.data(), evo_sigs.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(causal.data(), evo_causal.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(cls.data(), evo_classes.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(sts.data(), evo_states.p, nevo * 8, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaMemcpyAsync(stop.data(), evo_stopped.p, nevo * 4, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        out.assign(which.size(), EvolutionResult{});
        for (size_t i = 0; i < which.size(); ++i) {
            const uint32_t e = which[i];
            EvolutionResult& r = out[i];
            r.counts_only = true;
            r.num_classes = cls[e];
            r.n_states = sts[e];
            for (auto& q : evo_ranges[e].events) r.n_events += q.second - q.first;
            for (auto& q : evo_ranges[e].pairs) r.n_branchial += q.second - q.first;
            r.n_causal = causal[e];
            r.n_canonical_events = signatures ? sig[e] : r.n_events;
            r.truncated = stop[e] != 0;
        }
    }

    void finish_times() {
        flush_times();
        unsigned long long sv[8];
        HGX_CUDA_CHECK(cudaMemcpyAsync(sv, stats.p, sizeof(sv), cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        times.expand_bytes = sv[0];
        times.expand_hbm_bytes = sv[1];
        times.children = sv[2];
        times.wl_rounds = sv[3];
        times.warp_bytes = sv[4];
        times.warp_hbm_bytes = sv[5];
        times.warp_children = sv[6];
        times.warp_rounds = sv[7];
        times.launches = launches;
    }

    // ---- one level for every evolution in the frontier ---------------------------------------
    //
    // A single evolution under a state cap that the previous level's ratios (events per frontier
    // state, events per new state) place well inside this level's frontier is processed as two
    // frontier ranges in canonical order: a prefix sized to hold the cut, then the rest only if the
    // cap was not reached. Events, states and pairs keep their canonical numbering (the second range
    // follows the first), so the result is the one-pass result; the unexpanded tail is never counted.
    struct LevelHist {
        bool valid = false;
        double ev_per_state = 0, ev_per_new = 0;
        bool have_ok = false;   // have, stopped: evolution 0's classes, states and stopped flag
        unsigned long long have[2] = {0, 0};   // after the last range (one evolution)
        uint32_t stopped = 0;
    } hist;
    uint32_t sub_nf = 0;                           // next-frontier states written by earlier ranges
    uint64_t sub_ne = 0, sub_no = 0, sub_ev = 0, sub_new = 0;
    std::vector<uint64_t> sub_front;               // per evolution: next-frontier states so far
    std::vector<uint8_t> sub_part;                 // per evolution: in this level's frontier

    bool level(const RunOptions& opt) {
        const uint32_t F = frontier_size;
        if (F == 0) return false;
        const size_t nevo = h_evos.size();
        sub_nf = 0;
        sub_ne = sub_no = sub_ev = sub_new = 0;
        sub_front.assign(nevo, 0);
        sub_part.assign(nevo, 0);
        uint32_t P = F;
        const bool one_capped = nevo == 1 && !evo_done[0] && h_evos[0].max_states;
        if (one_capped && opt.level_split >= 2) {
            if (F > opt.level_split) P = static_cast<uint32_t>(opt.level_split);
        } else if (one_capped && opt.level_split == 0 && hist.valid && F >= 4096) {
            unsigned long long have[2] = {hist.have[0], hist.have[1]};
            if (!hist.have_ok) {
                readback(&have[0], evo_classes.p, 8);
                readback(&have[1], evo_states.p, 8);
                sync_st();
            }
            const uint64_t h = h_evos[0].quotient ? have[0] : have[1];
            const uint64_t remaining = h_evos[0].max_states > h ? h_evos[0].max_states - h : 0;
            const double need = double(remaining) * (h_evos[0].quotient ? hist.ev_per_new : 1.0);
            const double est = need / std::max(hist.ev_per_state, 1e-9) * 1.15 + 256;
            if (est < 0.8 * double(F)) P = static_cast<uint32_t>(est);
        }
        // the level's frontier ranges: [0, P), in up to four parts when the result streams (each
        // part's share of the result is copied out while the next computes), then [P, F)
        std::vector<std::pair<uint32_t, uint32_t>> parts;
        const uint32_t K = sr.on ? std::min<uint32_t>(4, std::max<uint32_t>(1, P / kStreamPartStates)) : 1;
        for (uint32_t j = 0; j < K; ++j)
            parts.emplace_back(uint32_t(uint64_t(P) * j / K), uint32_t(uint64_t(P) * (j + 1) / K));
        if (P < F) parts.emplace_back(P, F);
        bool cut = false;
        uint32_t stopped = 0;
        // evolution 0's stopped flag: from the last range's second sync, else read
        auto stopped_now = [&]() -> uint32_t {
            if (hist.have_ok) return hist.stopped;
            uint32_t v = 0;
            readback(&v, evo_stopped.p, 4);
            sync_st();
            return v;
        };
        for (size_t j = 0; j < parts.size(); ++j) {
            if (j > 0 && one_capped) {
                stopped = stopped_now();
                if (stopped) break;
            }
            level_range(opt, parts[j].first, parts[j].second);
        }
        if (parts.size() > 1 && one_capped) {
            stopped = stopped_now();
            // a level with a cut sends none of the evolution's new states on (the cut range has
            // sent none of its own; the earlier ranges' are dropped here)
            cut = stopped != 0;
            if (cut) {
                sub_nf = 0;
                sub_front[0] = 0;
            }
        }
        // the next level's estimate, from a level expanded whole
        if (P == F && sub_ev && sub_new) {
            hist.valid = true;
            hist.ev_per_state = double(sub_ev) / double(F);
            hist.ev_per_new = double(sub_ev) / double(sub_new);
        }
        // which evolutions still have a frontier
        for (size_t e = 0; e < nevo; ++e)
            if (sub_part[e] && !evo_done[e] && sub_front[e] == 0) {
                evo_done[e] = 1;
                finished.push_back(static_cast<uint32_t>(e));
            }
        std::swap(frontier, next_frontier);
        frontier_size = sub_nf;
        ne_bound = static_cast<uint32_t>(sub_ne);
        nocc_bound = static_cast<uint32_t>(sub_no);
        return frontier_size > 0;
    }

    // Frontier range [f0, f1) of the current level.
    void level_range(const RunOptions& opt, uint32_t f0, uint32_t f1) {
        const uint32_t F = f1 - f0;
        if (F == 0) return;
        const uint32_t R = rm.stride;
        const uint64_t items = uint64_t(F) * R;
        hist.have_ok = false;   // until this range's second sync
        if (items + 1 > 0xFFFFFFFFull) throw std::runtime_error("hgx: frontier too large for one level");
        const uint32_t NI = static_cast<uint32_t>(items);
        counts.ensure(NI, 0, st);
        item_ev.ensure(NI + 1, 0, st);
        item_cons.ensure(NI + 1, 0, st);
        item_prod.ensure(NI + 1, 0, st);
        item_fresh.ensure(NI + 1, 0, st);

        LevelArgs A;
        std::memset(&A, 0, sizeof(A));
        A.frontier = frontier.p + f0;
        A.n_frontier = F;
        A.rules_stride = R;
        A.counts = counts.p;
        A.item_ev = item_ev.p;
        A.item_cons = item_cons.p;
        A.item_prod = item_prod.p;
        A.item_fresh = item_fresh.p;
        A.work = work.p;
        A.level_max = level_max.p;
        A.ev_base = static_cast<uint32_t>(n_events);
        A.cons_base = static_cast<uint32_t>(n_cons);
        A.prod_base = static_cast<uint32_t>(n_edges);
        A.fresh_base = static_cast<uint32_t>(next_vertex);

        HGX_CUDA_CHECK(cudaMemsetAsync(work.p, 0, 8 * sizeof(uint32_t), st));
        HGX_CUDA_CHECK(cudaMemsetAsync(level_max.p, 0, 8 * sizeof(uint32_t), st));

        // ---- count
        const bool fwd = opt.forwarding != 0;
        A.fwd_mode = opt.forwarding;
        A.ev_keys = opt.event_keys;
        A.lane_vmax = F >= kLaneFullStates ? kLaneVMax : kLaneVMaxSmall;
        const Layout Lc = make_layout(ne_bound, nocc_bound, rm, LayoutKind::Count, fwd, kLaneJoinCap,
                                      opt.join_index != 0);
        fmode.ensure(F, 0, st);
        A.fmode = fmode.p;
        LaunchShape sc = warp_shape(k_count, Lc, F);
        tic();
        k_count<<<sc.grid, sc.block, sc.smem, st>>>(ptrs(), A, Lc);
        check_launch();
        toc(times.count);

        // ---- scans of the per-item sizes
        tic();
        k_item_sizes<<<grid_for(NI, 256), 256, 0, st>>>(ptrs(), A);
        check_launch();
        scan_multi({{item_ev.p, item_ev.p}, {item_cons.p, item_cons.p}, {item_prod.p, item_prod.p},
                    {item_fresh.p, item_fresh.p}}, NI);
        HGX_CUDA_CHECK(cudaMemsetAsync(evo_first_ev.p, 0xFF, h_evos.size() * 4, st));
        evo_frange.ensure(2 * h_evos.size(), 0, st);
        k_frontier_events<<<grid_for(F, 256), 256, 0, st>>>(ptrs(), A, evo_last_ev.p, evo_frange.p);
        check_launch();
        toc(times.scan);

        // ---- sync 1: level totals, per-evolution event ranges, exact frontier maxima
        const size_t nevo = h_evos.size();
        const size_t w1 = 5 + 4 * nevo;
        const unsigned long long* hs = sync_host(std::max<size_t>(w1, (7 * nevo + 9 + 1) / 2));
        k_sync1_pack<<<grid_for(std::max<size_t>(nevo, 1), 256), 256, 0, st>>>(
            item_ev.p, item_cons.p, item_prod.p, item_fresh.p, NI, level_max.p, evo_classes.p,
            evo_states.p, opt.event_keys ? evo_sigs.p : nullptr, evo_first_ev.p, evo_last_ev.p,
            static_cast<uint32_t>(nevo), d_sync);
        check_launch();
        sync_st();
        if (sr.on) stream_issue();   // the previous range's result chunk (its counts are here now)
        const uint32_t tot[6] = {uint32_t(hs[0]), uint32_t(hs[0] >> 32), uint32_t(hs[1]),
                                 uint32_t(hs[1] >> 32), uint32_t(hs[2]), uint32_t(hs[2] >> 32)};
        const uint32_t fmax_cnt = uint32_t(hs[3]);
        const uint32_t n_warp_states = uint32_t(hs[3] >> 32);   // 0: no warp-path launches
        const uint32_t fmax_nv = uint32_t(hs[4]);                // largest frontier vertex count
        std::vector<uint32_t> h_first(nevo), h_last(nevo);
        std::vector<unsigned long long> h_classes(hs + 5, hs + 5 + nevo),
            h_states_ev(hs + 5 + nevo, hs + 5 + 2 * nevo), h_sigs(hs + 5 + 2 * nevo, hs + 5 + 3 * nevo);
        for (size_t e = 0; e < nevo; ++e) {
            h_first[e] = uint32_t(hs[5 + 3 * nevo + e]);
            h_last[e] = uint32_t(hs[5 + 3 * nevo + e] >> 32);
        }
        auto h_states_now = [&](uint32_t e) { return static_cast<uint64_t>(h_states_ev[e]); };
        const uint32_t n_ev = tot[0], n_cons_lv = tot[1], n_prod = tot[2], n_fresh = tot[3];
        const uint32_t fmax_ne = tot[4], fmax_nocc = tot[5];
        if (uint64_t(n_events) + n_ev >= 0xFFFFFFF0ull || uint64_t(n_edges) + n_prod >= 0xFFFFFFF0ull ||
            uint64_t(next_vertex) + n_fresh >= 0xFFFFFFF0ull || uint64_t(n_cons) + n_cons_lv >= 0xFFFFFFF0ull)
            throw std::runtime_error("hgx: 32-bit id space exhausted (events, edges or vertices)");
        A.n_events = n_ev;

        // capacity
        grow_events(n_events + n_ev);
        ev_bmask.ensure(n_events + n_ev, n_events, st);
        ev_cons.ensure(n_cons + n_cons_lv, n_cons, st);
        ev_cprod.ensure(n_cons + n_cons_lv, n_cons, st);
        edge_creator.ensure(n_edges + n_prod, n_edges, st);
        flag_new.ensure(n_ev + 1, 0, st);
        scan_new.ensure(n_ev + 1, 0, st);
        flag_rep.ensure(n_ev + 1, 0, st);
        flag_front.ensure(n_ev + 1, 0, st);
        A.flag_new = flag_new.p;
        A.scan_new = scan_new.p;
        A.flag_rep = flag_rep.p;
        A.flag_front = flag_front.p;
        // tables: room for every event of the level plus every class seen
        bool any_cap = false;
        size_t grown_lo = nevo, grown_hi = 0;
        for (size_t e = 0; e < nevo; ++e) {
            if (evo_done[e] || h_first[e] == kNone) continue;
            if (h_evos[e].max_states) any_cap = true;
            const uint64_t lv = (h_last[e] >= h_first[e]) ? h_last[e] - h_first[e] : 0;
            const uint64_t need = h_classes[e] + lv + 1;
            bool grown = false;
            if (2 * need > h_evos[e].table_mask + 1) {
                regrow_table(static_cast<uint32_t>(e), need);
                grown = true;
            }
            // event signatures: every distinct one so far plus every event of this level
            const uint64_t need_s = h_sigs[e] + lv + 1;
            if (opt.event_keys && (!h_evos[e].sig_mask || 2 * need_s > h_evos[e].sig_mask + 1)) {
                regrow_region(h_evos[e].sig_off, h_evos[e].sig_mask, need_s);
                grown = true;
            }
            if (grown) {
                grown_lo = std::min(grown_lo, e);
                grown_hi = e + 1;
            }
        }
        upload_evos(grown_lo, grown_hi);

        // ---- expand: events, produced edges, children's WL hashes, table inserts
        //
        // An evolution whose state cap this level can reach is expanded in rounds over its
        // frontier range, in frontier (= canonical event) order, until the built events hold its
        // cut: every later event is dropped anyway, so the result is identical and the dropped
        // tail is never built. The other evolutions of the level are expanded whole in the first
        // round. Dedup stays exact because a round's events are selected only after every earlier
        // event of the evolution has been inserted. Unbuilt events of the last evolution in
        // frontier order are cut from the level; those of the others are voided (in-range ids,
        // never kept).
        uint32_t F_eff = F;
        bool tune = false, walk = false;   // join autotuner: measure this level / variant used
        uint32_t bucket = 0;
        if (n_ev) {
            const uint32_t mne = std::max<uint32_t>(fmax_ne, 1), mno = std::max<uint32_t>(fmax_nocc, 1);
            const Layout Ll = make_layout(std::min<uint32_t>(mne, kLaneEMax), mno, rm, LayoutKind::Lane, fwd,
                                          fmax_cnt);
            const Layout Lw = make_layout(mne, mno, rm, LayoutKind::Warp, fwd, kLaneJoinCap,
                                          opt.join_index != 0, fmax_nv);
            // lane kernel join: autotuned per bucket of children per frontier state (the walk
            // amortises its count-and-emit passes over many children per state)
            const uint64_t per_state = n_ev / std::max<uint32_t>(F, 1);
            while (bucket < 7 && (2ull << bucket) <= per_state) ++bucket;
            walk = per_state >= 32;
            if (opt.lane_join == 1) walk = false;
            else if (opt.lane_join == 2) walk = true;
            else {
                const uint32_t* tn = tuner.n[bucket];
                if (tn[0] >= 1 && tn[1] >= 1) walk = tuner.ns[bucket][1] < tuner.ns[bucket][0];
                else if (n_ev >= kTuneMinChildren) walk = tn[1] < tn[0];   // the less-sampled one
                tune = n_ev >= kTuneMinChildren;
            }
            // single-rule evolutions: batches of children cross parents (two parent regions per warp)
            Layout Ll2 = Ll;
            Ll2.bytes = Ll.bytes + (kLaneRegions - 1) * Ll.region_bytes;   // one batch per warp
            const bool cross = rm.stride == 1 && Ll2.bytes <= (kMaxDynSmem - 8192) / 2;
            LaunchShape sl = cross ? (walk ? (fwd ? warp_shape(k_expand_lanes2<true, kLaneRegions>, Ll2, F)
                                                  : warp_shape(k_expand_lanes2<true, kLaneRegions, false>, Ll2, F))
                                           : (fwd ? warp_shape(k_expand_lanes2<false, kLaneRegions>, Ll2, F)
                                                  : warp_shape(k_expand_lanes2<false, kLaneRegions, false>, Ll2, F)))
                                   : (walk ? warp_shape(k_expand<true, true>, Ll, F)
                                           : warp_shape(k_expand<true>, Ll, F));
            LaunchShape sw = warp_shape(k_expand<false>, Lw, n_ev);   // work units: slices
            auto expand = [&](uint32_t n_work) {
                A.f_begin = 0;
                A.f_end = n_work;
                HGX_CUDA_CHECK(cudaMemsetAsync(work.p + 1, 0, 2 * sizeof(uint32_t), st));
                tic(true);
                if (tune) HGX_CUDA_CHECK(cudaEventRecord(ev_a, st));
                // levels without forwarding run the lane kernel compiled without its paths
                if (cross && walk && fwd) k_expand_lanes2<true, kLaneRegions><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                else if (cross && walk) k_expand_lanes2<true, kLaneRegions, false><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                else if (cross && fwd) k_expand_lanes2<false, kLaneRegions><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                else if (cross) k_expand_lanes2<false, kLaneRegions, false><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                else if (walk) k_expand<true, true><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                else k_expand<true><<<sl.grid, sl.block, sl.smem, st>>>(ptrs(), A, Ll);
                check_launch();
                if (tune) HGX_CUDA_CHECK(cudaEventRecord(ev_b, st));
                toc(times.expand, true);
                ++times.expand_launches;
                if (walk) ++times.walk_launches;
                if (!n_warp_states) return;   // every state of the level is on the lane path
                tic();
                slice_off.ensure(uint64_t(n_work) + 1, 0, st);
                k_slice_counts<<<grid_for(n_work, 256), 256, 0, st>>>(A, n_work, slice_off.p);
                check_launch();
                scan(slice_off.p, slice_off.p, n_work);
                A.soff = slice_off.p;
                A.n_sw = n_work;
                k_expand<false><<<sw.grid, sw.block, sw.smem, st>>>(ptrs(), A, Lw);
                check_launch();
                A.soff = nullptr;
                toc(times.expand_warp);
            };
            struct Capped {
                uint32_t evo, lo, hi, built;
                uint64_t remaining, got, ev_built;
                bool open;
            };
            std::vector<Capped> capped;
            uint64_t avoidable = 0;
            for (size_t e = 0; e < nevo && any_cap; ++e) {
                if (evo_done[e] || h_first[e] == kNone || !h_evos[e].max_states) continue;
                const uint64_t have = h_evos[e].quotient ? h_classes[e] : h_states_now(e);
                const uint64_t remaining = h_evos[e].max_states > have ? h_evos[e].max_states - have : 0;
                const uint64_t lv = (h_last[e] >= h_first[e]) ? h_last[e] - h_first[e] : 0;
                if (lv <= remaining) continue;
                capped.push_back({static_cast<uint32_t>(e), 0, 0, 0, remaining, 0, 0, true});
                avoidable += lv - remaining;
            }
            if (capped.empty() || avoidable < opt.chunk_min) {
                A.frng = nullptr;
                expand(F);
                tic();
                k_select<<<grid_for(n_ev, 256), 256, 0, st>>>(ptrs(), A, 0, n_ev);
                check_launch();
                toc(times.select);
            } else {
                tune = false;   // rounds: several launches, no single measurement window
                std::vector<uint32_t> h_item(NI + 1), h_fr(2 * nevo);
                readback(h_item.data(), item_ev.p, (NI + 1) * 4);
                readback(h_fr.data(), evo_frange.p, 2 * nevo * 4);
                sync_st();
                auto fev = [&](uint32_t f) -> uint64_t { return h_item[uint64_t(f) * R]; };
                std::vector<uint8_t> is_capped(nevo, 0);
                for (Capped& c : capped) {
                    c.lo = c.built = h_fr[2 * c.evo];
                    c.hi = h_fr[2 * c.evo + 1];
                    is_capped[c.evo] = 1;
                }
                // the frontier ranges of a round, merged where adjacent, uploaded as A.frng
                std::vector<std::pair<uint32_t, uint32_t>> rng;
                auto run_ranges = [&](bool select) -> uint32_t {
                    std::sort(rng.begin(), rng.end());
                    std::vector<uint32_t> lo, off(1, 0);
                    for (const auto& r : rng) {
                        if (r.first >= r.second) continue;
                        if (!lo.empty() && lo.back() + (off.back() - off[off.size() - 2]) == r.first) {
                            off.back() += r.second - r.first;
                        } else {
                            lo.push_back(r.first);
                            off.push_back(off.back() + (r.second - r.first));
                        }
                    }
                    rng.clear();
                    const uint32_t n = static_cast<uint32_t>(lo.size()), total = off.back();
                    if (!total) return 0;
                    std::vector<uint32_t> buf(lo);
                    buf.insert(buf.end(), off.begin(), off.end());
                    frng.ensure(buf.size(), 0, st);
                    HGX_CUDA_CHECK(cudaMemcpyAsync(frng.p, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice, st));
                    A.frng = frng.p;
                    A.n_frng = n;
                    if (select) {
                        expand(total);
                        tic();
                        k_select_list<<<grid_for(uint64_t(total) * 32, 256), 256, 0, st>>>(ptrs(), A, total, evo_new.p);
                        check_launch();
                        toc(times.select);
                    }
                    return total;
                };
                evo_new.ensure(nevo, 0, st);
                std::vector<unsigned long long> h_new(nevo);
                for (size_t e = 0; e < nevo; ++e)
                    if (!evo_done[e] && h_first[e] != kNone && !is_capped[e])
                        rng.emplace_back(h_fr[2 * e], h_fr[2 * e + 1]);
                for (int round = 0;; ++round) {
                    std::vector<uint32_t> target(capped.size());
                    for (size_t i = 0; i < capped.size(); ++i) {
                        Capped& c = capped[i];
                        if (!c.open) continue;
                        // events to add: the new states still needed for the cut, scaled by the
                        // fraction of new classes seen so far (quotient mode), plus a margin
                        const uint64_t need = c.remaining + 1 - c.got;
                        uint64_t want = need;
                        if (h_evos[c.evo].quotient && c.ev_built) {
                            want = c.got ? need * c.ev_built / c.got : c.ev_built;
                            // margin: 1/20 for a lone capped evolution (a short round costs one more
                            // round), 1/4 with many (another round runs while any one is short)
                            want += want / (capped.size() == 1 ? 20 : 4) + 32;
                        }
                        if (round >= 12) want = UINT64_MAX;
                        const uint64_t goal = fev(c.built) + std::min<uint64_t>(want, UINT64_MAX / 2);
                        uint32_t a = c.built + 1, b = c.hi;   // first p in [a, b] with fev(p) >= goal
                        while (a < b) {
                            const uint32_t m = a + (b - a) / 2;
                            if (fev(m) >= goal) b = m; else a = m + 1;
                        }
                        target[i] = a;
                        rng.emplace_back(c.built, a);
                    }
                    HGX_CUDA_CHECK(cudaMemsetAsync(evo_new.p, 0, nevo * 8, st));
                    run_ranges(true);
                    readback(h_new.data(), evo_new.p, nevo * 8);
                    sync_st();
                    bool any_open = false;
                    for (size_t i = 0; i < capped.size(); ++i) {
                        Capped& c = capped[i];
                        if (!c.open) continue;
                        const uint64_t built = fev(target[i]) - fev(c.built);
                        c.got += h_evos[c.evo].quotient ? h_new[c.evo] : built;
                        c.ev_built += built;
                        c.built = target[i];
                        c.open = c.got <= c.remaining && c.built < c.hi;
                        any_open |= c.open;
                    }
                    if (!any_open) break;
                }
                for (const Capped& c : capped) {
                    if (c.built == c.hi) continue;
                    if (c.hi == F) F_eff = c.built;   // the level ends at the last built state
                    else rng.emplace_back(c.built, c.hi);
                }
                if (const uint32_t n_void = run_ranges(false)) {
                    k_void<<<grid_for(uint64_t(n_void) * 32, 256), 256, 0, st>>>(ptrs(), A, n_void);
                    check_launch();
                }
                A.frng = nullptr;
                A.n_frng = 0;
            }
            const uint32_t n_ev_eff = F_eff == F ? n_ev : [&] {
                uint32_t v = 0;
                readback(&v, item_ev.p + uint64_t(F_eff) * R, 4);
                sync_st();
                return v;
            }();
            A.n_events = n_ev_eff;
            if (n_ev_eff) {
                k_cprod<<<grid_for(n_ev_eff, 256), 256, 0, st>>>(ptrs(), A.ev_base, n_ev_eff);
                check_launch();
                if (opt.transitive_reduction) {
                    ev_anc.ensure(uint64_t(n_events) + n_ev_eff, n_events, st);
                    k_tr<<<grid_for(n_ev_eff, 256), 256, 0, st>>>(ptrs(), A.ev_base, n_ev_eff);
                    check_launch();
                }
            }

            // ---- cap / representatives over the events actually built
            const uint32_t ne2 = A.n_events;
            tic();
            if (any_cap) {
                scan(flag_new.p, scan_new.p, ne2);
                k_cut<<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
                check_launch();
            }
            k_rep<<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
            check_launch();
            scan_multi({{flag_rep.p, flag_rep.p}, {flag_front.p, flag_front.p}}, ne2);
            toc(times.select);
        } else {
            HGX_CUDA_CHECK(cudaMemsetAsync(flag_rep.p, 0, 4, st));
            HGX_CUDA_CHECK(cudaMemsetAsync(flag_front.p, 0, 4, st));
        }
        // frontier states whose events were built (all of them unless a chunked cut stopped early)
        A.n_frontier = F_eff;
        const uint32_t ne2 = A.n_events;
        bcount.ensure(uint64_t(ne2) + 1, 0, st);
        boff.ensure(uint64_t(ne2) + 1, 0, st);
        A.bcount = bcount.p;
        A.boff = boff.p;
        if (opt.branchial && ne2) {
            tic();
            k_bpairs<false><<<grid_for(uint64_t(F_eff) * 32, 256), 256, 0, st>>>(ptrs(), A);
            check_launch();
            if (fmax_ne > 63) {   // parents without position masks
                k_bpairs_walk<false><<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
                check_launch();
            }
            scan(bcount.p, boff.p, ne2);
            toc(times.branchial);
        } else {
            // no pairs this level: every offset is 0 (the per-evolution pair ranges read them)
            HGX_CUDA_CHECK(cudaMemsetAsync(boff.p, 0, (uint64_t(ne2) + 1) * 4, st));
        }

        // per-evolution ranges of this level (events kept, new states, branchial pairs)
        A.state_base = static_cast<uint32_t>(n_states);
        A.bbase = static_cast<uint32_t>(n_bpairs);
        const uint32_t* hs2 = reinterpret_cast<const uint32_t*>(sync_host((7 * nevo + 9 + 1) / 2));
        uint32_t* ds2 = reinterpret_cast<uint32_t*>(d_sync);
        if (ne2 || F_eff) {
            A.n_frontier = F;   // boundaries over the whole frontier; event ranges clamp to ne2
            k_evo_ranges<<<grid_for(F, 256), 256, 0, st>>>(ptrs(), A, evo_last_ev.p, ds2);
            check_launch();
            A.n_frontier = F_eff;
        }
        // ---- sync 2: new states, next frontier, branchial pairs, errors (behind the ranges)
        k_sync2_pack<<<1, 32, 0, st>>>(flag_rep.p, flag_front.p, boff.p, ne2, err.p, evo_classes.p,
                                       evo_states.p, evo_stopped.p, ds2 + 7 * nevo);
        check_launch();
        sync_st();
        if (nevo == 1) {
            hist.have[0] = hs2[7 * nevo + 4] | (uint64_t(hs2[7 * nevo + 5]) << 32);
            hist.have[1] = hs2[7 * nevo + 6] | (uint64_t(hs2[7 * nevo + 7]) << 32);
            hist.stopped = hs2[7 * nevo + 8];
            hist.have_ok = true;
        }
        const std::vector<uint32_t> h_rng(hs2, hs2 + 7 * nevo);
        const uint32_t* s2 = hs2 + 7 * nevo;
        if (tune) {
            float ms = 0;
            HGX_CUDA_CHECK(cudaEventElapsedTime(&ms, ev_a, ev_b));
            const double x = double(ms) * 1e6 / double(n_ev);
            double& avg = tuner.ns[bucket][walk ? 1 : 0];
            uint32_t& cnt = tuner.n[bucket][walk ? 1 : 0];
            avg = cnt ? 0.75 * avg + 0.25 * x : x;
            ++cnt;
        }
        if (s2[3] & kErrTrDepth)
            throw std::invalid_argument("transitive reduction supports evolutions of at most 64 levels");
        if (s2[3]) throw std::runtime_error("hgx: device error flags 0x" + std::to_string(s2[3]));
        const uint32_t n_new = s2[0], n_front = s2[1], n_b = s2[2];
        for (size_t e = 0; e < nevo; ++e) {
            if (evo_done[e] || h_first[e] == kNone) continue;
            const uint32_t* q = &h_rng[7 * e];
            // ranges must lie inside what this level produced
            if (q[0] > q[1] || q[1] > n_events + ne2 || q[2] > q[3] || q[3] > n_states + n_new ||
                q[4] > q[5] || q[5] > n_bpairs + n_b)
                throw std::runtime_error("hgx: inconsistent per-evolution ranges at a level");
            if (q[1] > q[0]) evo_ranges[e].events.emplace_back(q[0], q[1]);
            if (q[3] > q[2]) evo_ranges[e].states.emplace_back(q[2], q[3]);
            if (opt.branchial && q[5] > q[4]) evo_ranges[e].pairs.emplace_back(q[4], q[5]);
        }

        grow_states(n_states + n_new);
        new_state_event.ensure(n_new, 0, st);
        next_frontier.ensure(uint64_t(sub_nf) + n_front, sub_nf, st);
        const uint64_t max_ne = uint64_t(fmax_ne) + rm.grow_e, max_no = uint64_t(fmax_nocc) + rm.grow_o;
        const uint64_t rec_words = max_ne + (max_ne + 3) / 4 + max_no;
        arena.ensure(arena_words + uint64_t(n_new) * rec_words, arena_words, st);
        bpairs.ensure(2ull * (n_bpairs + n_b), 2ull * n_bpairs, st);
        A.state_base = static_cast<uint32_t>(n_states);
        A.new_state_event = new_state_event.p;
        A.next_frontier = next_frontier.p + sub_nf;
        A.bpairs = bpairs.p;
        A.bbase = static_cast<uint32_t>(n_bpairs);
        if (ne2) {
            tic();
            k_assign<<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
            check_launch();
            k_outstate<<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
            check_launch();
            if (opt.event_keys) {
                ev_sig.ensure(n_events + ne2, n_events, st);
                for (int pass = 0; pass < 2; ++pass) {
                    k_evsig<<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A, pass);
                    check_launch();
                }
            }
            if (n_new) {
                // lanes per state: 8 up to 16-edge parents (four states per warp pass share its
                // fixed cost; measured faster than 16 lanes and one pass), else 32
                if (fmax_ne <= 16)   // 8-lane segments, two passes over a 9-16-edge parent
                    k_materialize<8><<<grid_for(n_new, 256), 256, 0, st>>>(ptrs(), A, n_new);
                else
                    k_materialize<32><<<grid_for(n_new, 256), 256, 0, st>>>(ptrs(), A, n_new);
                check_launch();
            }
            toc(times.materialize);
        }
        if (opt.branchial && n_b) {
            tic();
            // pair offsets are absolute: shift by the running total
            A.boff = boff.p;
            A.bpairs = bpairs.p + 2ull * n_bpairs;
            k_bpairs<true><<<grid_for(uint64_t(F_eff) * 32, 256), 256, 0, st>>>(ptrs(), A);
            check_launch();
            if (fmax_ne > 63) {
                k_bpairs_walk<true><<<grid_for(ne2, 256), 256, 0, st>>>(ptrs(), A);
                check_launch();
            }
            toc(times.branchial);
        }

        // the evolutions of this range and their next-frontier counts (from sync 2)
        for (size_t e = 0; e < nevo; ++e)
            if (!evo_done[e] && h_first[e] != kNone) {
                sub_part[e] = 1;
                sub_front[e] += h_rng[7 * e + 6];
            }

        // advance (id ranges of produced edges / fresh vertices / consumed lists were reserved for
        // the whole level; a chunked cut leaves the unbuilt tail of those ranges unused)
        n_events += ne2;
        n_cons += n_cons_lv;
        n_edges += n_prod;
        next_vertex += n_fresh;
        n_states += n_new;
        n_bpairs += n_b;
        arena_words += uint64_t(n_new) * rec_words;   // host bound >= the device bump pointer
        sub_nf += n_front;
        sub_ne = std::max(sub_ne, max_ne);
        sub_no = std::max(sub_no, max_no);
        sub_ev += n_ev;
        sub_new += n_new;
        if (sr.on && !evo_done[0] && h_first[0] != kNone) stream_prep(&h_rng[0], max_ne, max_no);
    }
};

// ==========================================================================================

Engine::Engine(int device) : impl_(new Impl(device)) {}
Engine::~Engine() = default;

std::vector<EvolutionResult> Engine::run(const std::vector<EvolutionSpec>& specs, const RunOptions& opt) {
    Impl& I = *impl_;
    BudgetScope scope(&I.budget);
    HGX_CUDA_CHECK(cudaSetDevice(I.device));
    I.reset();
    std::vector<const EvolutionSpec*> ptrs;
    for (const auto& s : specs) ptrs.push_back(&s);
    const std::vector<uint32_t> ids = I.admit_many(ptrs);
    I.stream_begin(opt);
    while (I.level(opt)) {}
    std::vector<EvolutionResult> out;
    if (!opt.readback) {
        I.read_counts(ids, out, opt.event_keys != 0);
    } else if (ids.size() == 1) {
        EvolutionResult r;
        if (I.sr.on && !I.sr.failed) r = I.finalize_streamed();
        if (!r.flat) {   // not streamed, or a block had no room: the whole result at once
            if (I.sr.on) I.stream_abort();
            r = I.finalize_single(opt);
            if (Impl::stream_eligible(opt, 1)) I.stream_hints(r.flat->count);
        }
        out.push_back(std::move(r));
    } else {
        out = I.finalize_many(ids, opt);
    }
    I.finish_times();
    return out;
}

void Engine::reset() {
    BudgetScope scope(&impl_->budget);
    impl_->reset();
}
uint32_t Engine::admit(const EvolutionSpec& spec) {
    BudgetScope scope(&impl_->budget);
    return impl_->admit(spec);
}
std::vector<uint32_t> Engine::admit(const std::vector<EvolutionSpec>& specs) {
    BudgetScope scope(&impl_->budget);
    std::vector<const EvolutionSpec*> ptrs;
    for (const auto& s : specs) ptrs.push_back(&s);
    return impl_->admit_many(ptrs);
}
bool Engine::step(const RunOptions& opt) {
    BudgetScope scope(&impl_->budget);
    return impl_->level(opt);
}
void Engine::set_device_limit(uint64_t bytes) { impl_->budget.limit = bytes; }
uint64_t Engine::device_limit() const { return impl_->budget.limit; }
std::vector<uint32_t> Engine::take_finished() {
    std::vector<uint32_t> f;
    f.swap(impl_->finished);
    return f;
}
EvolutionResult Engine::collect(uint32_t evo, const RunOptions& opt) {
    if (evo >= impl_->h_evos.size()) throw std::invalid_argument("collect: unknown evolution id");
    return std::move(collect(std::vector<uint32_t>{evo}, opt)[0]);
}
std::vector<EvolutionResult> Engine::collect(const std::vector<uint32_t>& evos, const RunOptions& opt) {
    BudgetScope scope(&impl_->budget);
    for (uint32_t evo : evos)
        if (evo >= impl_->h_evos.size()) throw std::invalid_argument("collect: unknown evolution id");
    if (opt.readback) return impl_->finalize_many(evos, opt);
    std::vector<EvolutionResult> out;
    impl_->read_counts(evos, out, opt.event_keys != 0);
    return out;
}
uint32_t Engine::active() const {
    uint32_t n = 0;
    for (uint8_t d : impl_->evo_done) n += d ? 0 : 1;
    return n;
}
uint64_t Engine::device_bytes_in_use() const {
    const Impl& I = *impl_;
    return I.arena.bytes() + I.st_off.bytes() * 2 + I.st_ne.bytes() * 5 + I.edge_creator.bytes() +
           I.ev_in.bytes() * 8 + I.ev_hash.bytes() + I.ev_cons.bytes() * 2 + I.tab_keys.bytes() +
           I.tab_vals.bytes() + I.bpairs.bytes();
}
uint64_t Engine::estimate_bytes(const EvolutionSpec& spec) {
    // Level by level: the largest state at depth d has E_d = E_0 + d * max(0, rhs - lhs) edges
    // (O_d occurrences likewise); a state has at most sum over rules of E_d! / (E_d - L)! matches
    // (ordered edge-injective tuples); states are bounded by the cap (2^22 when uncapped), events
    // by that bound and by 64 per state, branchial pairs by 16 per event. Bytes per state, event
    // and pair follow the engine's arrays, with 1.5x growth slack.
    auto sat_mul = [](uint64_t a, uint64_t b) -> uint64_t {
        return (a && b > UINT64_MAX / a) ? UINT64_MAX : a * b;
    };
    uint64_t e0 = 0, o0 = 0;
    for (const auto& r : spec.roots) {
        uint64_t o = 0;
        for (const auto& e : r) o += e.size();
        e0 = std::max<uint64_t>(e0, r.size());
        o0 = std::max(o0, o);
    }
    int64_t grow_e = 0, grow_o = 0;
    uint64_t lhs_max = 1, rhs_max = 0;
    for (const auto& r : spec.rules) {
        int64_t lo = 0, ro = 0;
        for (const auto& e : r.lhs) lo += static_cast<int64_t>(e.size());
        for (const auto& e : r.rhs) ro += static_cast<int64_t>(e.size());
        grow_e = std::max<int64_t>(grow_e, static_cast<int64_t>(r.rhs.size()) - static_cast<int64_t>(r.lhs.size()));
        grow_o = std::max<int64_t>(grow_o, ro - lo);
        lhs_max = std::max<uint64_t>(lhs_max, r.lhs.size());
        rhs_max = std::max<uint64_t>(rhs_max, r.rhs.size());
    }
    const uint64_t cap = spec.max_states ? spec.max_states : (1ull << 22);
    uint64_t frontier = spec.roots.size(), states = spec.roots.size(), events = 0;
    for (uint32_t d = 0; d < spec.steps && frontier && states < cap; ++d) {
        const uint64_t E = e0 + d * static_cast<uint64_t>(grow_e);
        uint64_t m = 0;
        for (const auto& r : spec.rules) {
            uint64_t p = 1;
            for (uint64_t k = 0; k < r.lhs.size(); ++k) p = sat_mul(p, E > k ? E - k : 0);
            m = std::min<uint64_t>(UINT64_MAX - p, m) + p;
        }
        const uint64_t ev = sat_mul(frontier, m);
        events = std::min<uint64_t>(UINT64_MAX - ev, events) + ev;
        const uint64_t fresh = std::min(cap - states, ev);
        states += fresh;
        frontier = fresh;
    }
    events = std::min(events, 64 * states);
    const uint64_t E = e0 + spec.steps * static_cast<uint64_t>(grow_e);
    const uint64_t O = o0 + spec.steps * static_cast<uint64_t>(grow_o);
    const uint64_t per_state = 56 + 4 * (E + (E + 3) / 4 + O) + 48;   // SoA + record + table
    const uint64_t per_event = 112 + 8 * lhs_max + 4 * rhs_max + 16 * 8;   // + branchial pairs
    const uint64_t total = states * per_state + events * per_event;
    return total + total / 2 + (1ull << 20);
}
cudaStream_t Engine::stream() const { return impl_->st; }
void Engine::set_timing(int level) { impl_->timing = level; }
const StageTimes& Engine::times() const { return impl_->times; }
void Engine::sync() { HGX_CUDA_CHECK(cudaStreamSynchronize(impl_->st)); }

}  // namespace hgx

// ==========================================================================================
// Allocation-free state hashing (hgx_hash_states_noalloc).
//
// For callers that cannot call cudaMalloc: code running under a runtime that owns the device's
// memory (a framework's caching allocator, a database or serving process with a fixed device
// budget) where a foreign allocation breaks its accounting or fails outright, and code on a
// latency-critical path where cudaMalloc's implicit device synchronisation is not acceptable.
// They pass their own device buffers for inputs and outputs; the only scratch this needs -- the
// dedup table, a work counter and an error word -- lives in the file-scope array below, which
// every GPU that loads this library holds (kNoAllocScratchBytes) until the process exits.
// ==========================================================================================

namespace hgx {
namespace {

constexpr uint32_t kNoAllocMaxStates = 1u << 19;               // table load factor <= 1/2
constexpr uint64_t kNoAllocSlots = 1ull << 20;                 // table capacity (power of two)
constexpr uint64_t kNoAllocKeyBytes = (kNoAllocSlots + 1) * 8;
constexpr uint64_t kNoAllocValBytes = (kNoAllocSlots + 1) * 4;
constexpr uint64_t kNoAllocScratchBytes = kNoAllocKeyBytes + kNoAllocValBytes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The device address of g_noalloc_scratch, per device. In host code the symbol's name is only a
// host-side handle, not a device address, so it is resolved once per device (with that device
// current) through cudaGetSymbolAddress and the kernels are given the resolved pointer.
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};

hgx_status noalloc_fail(hgx_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

__global__ void k_noalloc_classes(DevPtrs P, DevEvo ev, const uint64_t* hash, uint32_t n,
                                  uint32_t* cls) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        cls[i] = table_lookup(P, ev, hash[i]);
}

// Warp per state: WL hash into hash[i], then insert (hash, i) into the table (smallest i wins).
__global__ void __launch_bounds__(256) k_noalloc_hash(DevPtrs P, DevEvo ev, uint32_t n,
                                                     uint32_t* work, uint64_t* hash, Layout L) {
    extern __shared__ __align__(16) char smem[];
    char* sm = smem + (threadIdx.x >> 5) * L.bytes;
    const uint32_t lane = lane_id();
    while (true) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(work, 1u);
        i = __shfl_sync(0xFFFFFFFFu, i, 0);
        if (i >= n) break;
        const Parent pa = load_parent(P, L, sm, i);
        uint8_t* car = smp<uint8_t>(sm, L.o_car);
        uint16_t* cvo = smp<uint16_t>(sm, L.o_cvo);
        const uint8_t* pear = smp<uint8_t>(sm, L.o_pear);
        const uint16_t* pevo = smp<uint16_t>(sm, L.o_pevo);
        for (uint32_t e = lane; e < pa.ne; e += 32) { car[e] = pear[e]; cvo[e] = pevo[e]; }
        __syncwarp();
        WlInfo info;
        const uint64_t h = warp_wl(L, sm, pa.ne, pa.nvp, info);
        if (lane == 0) {
            hash[i] = h;
            table_insert(P, ev, h, i);
        }
        __syncwarp();
    }
}

}  // namespace
}  // namespace hgx

extern "C" HGX_API hgx_status hgx_hash_states_noalloc(
    const uint32_t* d_records, const uint64_t* d_offsets, const uint32_t* d_num_edges,
    const uint32_t* d_num_occ, uint32_t n_states, uint32_t max_edges, uint32_t max_occ,
    uint64_t* d_hash, uint32_t* d_class, void* stream) {
    using namespace hgx;
    try {
        if (n_states > kNoAllocMaxStates)
            return noalloc_fail(HGX_ERR_CAPACITY,
                                "hgx_hash_states_noalloc: " + std::to_string(n_states) +
                                    " states exceed the maximum of " +
                                    std::to_string(kNoAllocMaxStates) + " per call");
        if (n_states == 0) return HGX_OK;
        if (!d_records || !d_offsets || !d_num_edges || !d_num_occ || !d_hash || !d_class)
            return noalloc_fail(HGX_ERR_INVALID, "hgx_hash_states_noalloc: null device pointer");
        if (max_edges == 0 || max_occ == 0)
            return noalloc_fail(HGX_ERR_INVALID, "hgx_hash_states_noalloc: max_edges and max_occ must be > 0");
        RuleMax rm;
        rm.arity = kMaxArity;
        const Layout L = make_layout(max_edges, max_occ, rm, LayoutKind::Warp);
        if (L.bytes > kMaxDynSmem)
            return noalloc_fail(HGX_ERR_CAPACITY,
                                "hgx_hash_states_noalloc: states of this size exceed shared memory");
        int dev = 0;
        HGX_CUDA_CHECK(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) return noalloc_fail(HGX_ERR_INVALID, "device index out of range");
        unsigned char* base = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_noalloc_mu);
            if (!g_noalloc_ptr[dev]) {   // first call on this device: resolve the scratch address
                void* p = nullptr;
                const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
                if (e != cudaSuccess || !p)
                    return noalloc_fail(HGX_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") +
                                                          cudaGetErrorString(e));
                HGX_CUDA_CHECK(cudaFuncSetAttribute(k_noalloc_hash,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    static_cast<int>(kMaxDynSmem)));
                g_noalloc_ptr[dev] = p;
            }
            base = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
        }
        unsigned long long* keys = reinterpret_cast<unsigned long long*>(base);
        uint32_t* vals = reinterpret_cast<uint32_t*>(base + kNoAllocKeyBytes);
        uint32_t* counters = reinterpret_cast<uint32_t*>(base + kNoAllocKeyBytes + kNoAllocValBytes);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // a table of at least twice the states; the array keeps the previous call's contents,
        // so the used region and the counters are cleared first
        uint64_t cap = 256;
        while (cap < 2ull * n_states) cap <<= 1;
        DevEvo ev;
        std::memset(&ev, 0, sizeof(ev));
        ev.table_off = 0;
        ev.table_mask = cap - 1;
        // slots [0, cap) plus the key-0 slot at index cap
        HGX_CUDA_CHECK(cudaMemsetAsync(keys, 0, (cap + 1) * 8, st));
        HGX_CUDA_CHECK(cudaMemsetAsync(vals, 0xFF, (cap + 1) * 4, st));
        HGX_CUDA_CHECK(cudaMemsetAsync(counters, 0, 8, st));
        DevPtrs P;
        std::memset(&P, 0, sizeof(P));
        P.arena = const_cast<uint32_t*>(d_records);
        P.st_off = const_cast<uint64_t*>(d_offsets);
        P.st_ne = const_cast<uint32_t*>(d_num_edges);
        P.st_nocc = const_cast<uint32_t*>(d_num_occ);
        P.tab_keys = keys;
        P.tab_vals = vals;
        P.err = counters + 1;
        const uint32_t wpb = static_cast<uint32_t>(std::min<size_t>(8, std::max<size_t>(1, (96 * 1024) / L.bytes)));
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((n_states + wpb - 1) / wpb, kNumSMs * 4));
        k_noalloc_hash<<<grid, 32 * wpb, L.bytes * wpb, st>>>(P, ev, n_states, counters, d_hash, L);
        HGX_CUDA_CHECK(cudaGetLastError());
        k_noalloc_classes<<<(n_states + 255) / 256, 256, 0, st>>>(P, ev, d_hash, n_states, d_class);
        HGX_CUDA_CHECK(cudaGetLastError());
        uint32_t err = 0;
        HGX_CUDA_CHECK(cudaMemcpyAsync(&err, counters + 1, 4, cudaMemcpyDeviceToHost, st));
        HGX_CUDA_CHECK(cudaStreamSynchronize(st));
        if (err)
            return noalloc_fail(HGX_ERR_CAPACITY, "hgx_hash_states_noalloc: a state exceeds max_edges / "
                                                  "max_occ or its record is inconsistent (an arity "
                                                  "outside 1..16, or arities not adding up to its "
                                                  "occurrence count), or the table overflowed (flags " +
                                                  std::to_string(err) + ")");
        return HGX_OK;
    } catch (const std::exception& e) {
        return noalloc_fail(HGX_ERR_CUDA, e.what());
    }
}
