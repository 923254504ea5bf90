// Shared device/host definitions for the B200 multiway evolution step.
//
// Integer hash primitives restate common/include/hgcommon/core.hpp:47-87 of the reference
// (FNV-1a step, splitmix64 finaliser) and the reserved empty-state hash (core.hpp:169). They
// must agree bit for bit with the reference because every state identity is built from them.
#pragma once
#include <cstdint>
#include <cstdio>

#ifdef __CUDACC__
#define HGX_HD __host__ __device__ __forceinline__
#define HGX_NOINLINE __host__ __device__ __noinline__
#else
#define HGX_HD inline
#define HGX_NOINLINE inline
#endif

namespace hgx {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ULL;
constexpr uint64_t kFnvPrime = 0x100000001b3ULL;
constexpr uint64_t kEmptyStateHash = 0x9E3779B97F4A7C15ULL;
constexpr uint32_t kWlMaxRounds = 100;

// Limits of the rule representation (the reference's MAX_PATTERN_EDGES / MAX_ARITY /
// MAX_VARS, common/include/hgcommon/core.hpp:42-44).
constexpr int kMaxPatternEdges = 16;
constexpr int kMaxArity = 16;
constexpr int kMaxVars = 32;
constexpr int kMaxSideVars = 64;   // total positions over one rule side (16 edges x 4 avg)

// Lane-per-child WL: a parent with at most kLaneEMax edges whose children have at most
// kLaneVMax vertices is expanded with one child per lane -- on a level whose frontier fills the
// GPU with lane-kernel warps (kLaneFullStates states, one warp per parent in every warp slot of
// 148 SMs x 4 blocks x 8 warps). A smaller level takes the lane path only for children of at
// most kLaneVMaxSmall vertices: a lane's WL work grows with the square of the child's vertices,
// and the warp-per-child path spreads a larger child over the lanes and a small level over more
// warps (256 evolutions of the random batch, one per call: 439 -> 326 ms; the 1024-evolution
// batch at cap 4,096: 118 -> 113 ms); on full levels the lane path stays faster (the batch at cap
// 65,536: 628 ms either way, 805 ms with the lower limit on every level), and 9-vertex children
// run 7x faster one per lane either way.
constexpr int kLaneVMax = 32;
constexpr int kLaneVMaxSmall = 12;
constexpr uint32_t kLaneFullStates = 148 * 4 * 8;
constexpr int kLaneEMax = 64;
constexpr int kLaneNMax = 64;    // neighbour entries a lane sorts for one vertex

// Match forwarding: at most this many delta matches per state (else the state is re-joined), and
// rules of at most 4 LHS edges (a match's canonical key packs 4 positions of 16 bits).
constexpr uint32_t kFwdCap = 256;
constexpr uint32_t kFwdMaxLhs = 4;

// States with more vertex occurrences than this number their vertices through a hash table.
// Lane-parallel join: states of at most this many edges (positions fit one byte), rules of at
// most kLaneJoinLhs LHS edges (four positions pack into one word), and per (state, rule) at most
// kLaneJoinCap matches staged in shared memory by the expand kernel.
constexpr uint32_t kLaneJoinLhs = 4, kLaneJoinCap = 256;
constexpr uint32_t kHashOccMin = 96;

// Join indices: states of more than kJoinIndexMin edges staged for the warp join carry a vertex
// index and, when their edges fall in at most kSigBuckets signatures, a signature index.
constexpr uint32_t kJoinIndexMin = 96;
constexpr uint32_t kSigBuckets = 16;

// (Writing the multiply by the prime 2^40 + 0x1b3 as a shift and a 32-bit multiply measured
// slower on the lane expand kernel: 6.72 -> 6.79 ms per C2 evolution.)
HGX_HD uint64_t fnv(uint64_t h, uint64_t x) { return (h ^ x) * kFnvPrime; }

HGX_HD uint64_t smix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Rule flag: the RHS edges form one connected hypergraph holding every LHS variable. Then a child
// is connected exactly when its parent is: every component left after removing the matched edges
// touches a matched vertex, and the produced edges join all of those.
constexpr uint8_t kRuleRhsJoinsLhs = 1u << 0;

// A rewrite rule as the kernels read it: one fixed-size record, copied to shared memory by
// the warp that applies it. `sched` is the binding order of the LHS positions; matches are
// enumerated in lexicographic order of their edges' state positions taken in that order.
struct DevRule {
    uint8_t n_lhs, n_rhs, n_fresh, lhs_total, rhs_total;
    uint8_t flags;           // kRule* bits
    uint8_t rhs_uni;         // the arity every RHS edge has (0 when they differ)
    uint8_t pad;
    uint32_t new_mask;       // variables that occur only on the RHS
    uint8_t lhs_ar[kMaxPatternEdges], lhs_off[kMaxPatternEdges];
    uint8_t rhs_ar[kMaxPatternEdges], rhs_off[kMaxPatternEdges];
    uint8_t sched[kMaxPatternEdges];
    uint8_t fresh_rank[kMaxVars];   // n-th fresh variable -> n (ascending variable order)
    uint8_t lhs_vars[kMaxSideVars];
    uint8_t rhs_vars[kMaxSideVars];
    uint8_t rhs_pos_edge[kMaxSideVars];   // RHS position -> its edge
};
static_assert(sizeof(DevRule) % 4 == 0, "rule record must be word aligned");

// Per-evolution bookkeeping the kernels read.
struct DevEvo {
    uint32_t rule_begin;     // first rule of this evolution in the rule table
    uint32_t rule_count;
    uint32_t steps;          // expansion budget: states at depth < steps are expanded
    uint32_t quotient;       // 1 = expand each WL class once (at its shortest depth)
    uint64_t table_off;      // slot offset of this evolution's dedup table
    uint64_t table_mask;     // capacity - 1 (power of two); slot mask+1 holds key 0
    uint64_t max_states;     // 0 = unlimited
    uint64_t sig_off;        // event-signature table (event canonicalisation), same layout;
    uint64_t sig_mask;       // sig_mask == 0: not allocated
};

// Event signature keys (hgcommon EventSignatureKeys bits, common/include/hgcommon/event_core.hpp:30-37)
// that this path computes: the edge-rank keys (1 << 4, 1 << 5) need an exact canonical labelling.
constexpr uint32_t kEvKeyInput = 1u << 0, kEvKeyOutput = 1u << 1, kEvKeyStep = 1u << 2,
                   kEvKeyRule = 1u << 3, kEvKeysSupported = 0xFu;

// Signature of one event from the selected keys, in the key order of hgcommon::event_signature
// (common/include/hgcommon/event_core.hpp:64-84); 0 and the bare offset are reserved and map to 1.
HGX_HD uint64_t event_signature(uint32_t keys, uint64_t in_hash, uint64_t out_hash,
                                       uint32_t step, uint32_t rule) {
    uint64_t sig = kFnvOffset;
    if (keys & kEvKeyInput) sig = fnv(sig, in_hash);
    if (keys & kEvKeyOutput) sig = fnv(sig, out_hash);
    if (keys & kEvKeyStep) sig = fnv(sig, static_cast<uint64_t>(step));
    if (keys & kEvKeyRule) sig = fnv(sig, static_cast<uint64_t>(rule));
    return (sig == 0 || sig == kFnvOffset) ? 1 : sig;
}

// Device-side error channel (typed, host-visible; never a trap).
enum ErrorBits : uint32_t {
    kErrTableFull = 1u << 0,
    kErrStateTooLarge = 1u << 1,
    kErrArenaFull = 1u << 2,
    kErrBadRule = 1u << 3,
    kErrTrDepth = 1u << 4,       // transitive reduction past 64 levels
    kErrJoinCount = 1u << 5,     // a state's matches differ between the count and expand passes
};

}  // namespace hgx

#define HGX_CUDA_CHECK(expr)                                                                 \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) {                                                             \
            throw ::hgx::CudaError(_e, #expr, __FILE__, __LINE__);                           \
        }                                                                                    \
    } while (0)
