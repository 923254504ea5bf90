// Kernels of one level-synchronous multiway step (sm_100a).
//
// A step takes the frontier (states to expand, from any number of independent evolutions) to
// the next frontier:
//
//   count      warp per frontier state: enumerate every rule's matches, count them
//   scan       exclusive scan of the per-(state, rule) counts -> event / edge / vertex ids
//   expand     warp per frontier state: enumerate again; per match write the event, mint the
//              produced edges, build the child in shared memory, WL-hash it and insert the
//              hash into the evolution's dedup table (first arrival wins via atomicMin)
//   select     thread per event: is the child the first arrival of its WL class? cap check
//   assign     thread per event: representative children become states / next frontier
//   materialize warp per new state: write its edge record (ids, arities, vertices)
//   branchial  warp per frontier state: event pairs of one input state sharing a consumed edge
//
// Everything is integer; there is no floating point on this path.
#pragma once
#include "common.cuh"

namespace hgx {

// All device arrays of an engine, by value into every kernel.
struct DevPtrs {
    // rules / evolutions
    const DevRule* rules;
    const DevEvo* evos;
    // states (SoA, indexed by global state id)
    uint64_t* st_off;       // word offset of the state's edge record in `arena`
    uint32_t* st_ne;        // edges
    uint32_t* st_nocc;      // vertex occurrences (sum of arities)
    uint32_t* st_evo;
    uint32_t* st_depth;
    uint32_t* st_event;     // arrival (event or root pseudo-event) that created it
    uint32_t* st_ev0;       // first event of the state's expansion (single-rule evolutions)
    uint32_t* st_evn;       // events of the state's expansion
    uint32_t* st_nv;        // distinct vertices of the state
    uint64_t* st_hash;
    uint32_t* arena;        // per-state records: ids[ne] | arity bytes[ceil(ne/4) words] | verts[nocc]
    unsigned long long* arena_top;
    uint64_t arena_cap;
    // edges (global ids)
    uint32_t* edge_creator; // producing event, kNone for initial edges
    // events (arrival ids; roots occupy pseudo-event slots with ev_in == kNone)
    uint32_t* ev_in;
    uint32_t* ev_rule;
    uint32_t* ev_coff;      // offset of the consumed-edge list in ev_cons / ev_cprod
    uint32_t* ev_prod;      // id of the first produced edge (RHS order, consecutive)
    uint32_t* ev_fresh;     // first fresh vertex id (consecutive, ascending variable order)
    uint32_t* ev_out;       // output state (the class representative in quotient mode)
    uint8_t*  ev_kept;      // 0 when a state cap cut the event off
    uint64_t* ev_hash;      // WL hash of the output state
    uint32_t* ev_nv;        // distinct vertices of the output state
    uint32_t* ev_cons;      // consumed edge ids, pattern order
    uint32_t* ev_cprod;     // producer event of each consumed edge
    uint32_t* state_of_arrival;
    // dedup tables (all evolutions, each at its own offset)
    unsigned long long* tab_keys;
    uint32_t* tab_vals;
    // per-evolution counters
    unsigned long long* evo_classes;   // WL classes seen so far
    unsigned long long* evo_causal;    // causal triples of the kept events so far
    unsigned long long* evo_states;    // states recorded so far
    uint32_t* evo_cut;                 // first event cut off by the cap this level (kNone = none)
    uint32_t* evo_first_ev;            // first event of the evolution in this level
    uint32_t* evo_stopped;
    // transitive reduction: per event, bit d set = an event at level d is a proper causal
    // ancestor (levels < 64; an event's ancestors lie on its input state's history chain)
    unsigned long long* ev_anc;
    // per event: the parent positions it consumed as a bit mask for the branchial test, or 0 when
    // the parent has more than 63 edges (compare edge ids); bit 63 alone: the event is not kept
    unsigned long long* ev_bmask;
    // event canonicalisation: per event its signature; per evolution the distinct signatures
    unsigned long long* ev_sig;
    unsigned long long* evo_sigs;
    // errors
    uint32_t* err;
    // expand-kernel counters, [0..3] lane-per-child kernel, [4..7] warp-per-child kernel:
    // bytes by the per-stage figures (join + rewrite + WL + dedup as separate streams), bytes the
    // fused kernel must move to/from HBM, children hashed, WL refinement rounds run
    unsigned long long* stats;
};

// Per-level parameters.
struct LevelArgs {
    const uint32_t* frontier;   // state ids
    uint32_t n_frontier;
    uint32_t rules_stride;      // R: item (f, r) = f * R + r
    uint32_t* counts;           // [F*R] matches per item
    uint32_t* item_ev;          // [F*R+1] exclusive scans
    uint32_t* item_cons;
    uint32_t* item_prod;
    uint32_t* item_fresh;
    uint32_t ev_base, cons_base, prod_base, fresh_base;   // level bases
    uint32_t n_events;          // events minted this level
    uint32_t f_begin, f_end;    // frontier range the expand kernel works on
    // if set: work index w in [f_begin, f_end) is a position inside n_frng frontier ranges,
    // frng[0, n) = first positions, frng[n, 2n+1) = exclusive prefix of the range lengths
    const uint32_t* frng;
    uint32_t n_frng;
    // warp-per-child kernel: exclusive scan over the n_sw work indices of their parents' slice
    // counts (soff[n_sw] = total); a slice is a run of slice_size(children) consecutive children
    const uint32_t* soff;
    uint32_t n_sw;
    uint8_t* fmode;             // [F] bit 0: children hashed lane-per-child; bit 1: forwarding
    uint32_t fwd_mode;          // 0 off, 1 every eligible state, 2 states with >= 48 edges
    uint32_t ev_keys;           // event signature keys (0 = no event canonicalisation)
    uint32_t lane_vmax;         // largest child (vertices) of this level the lane path takes
    uint32_t* work;             // work-queue counters
    // select / assign
    uint32_t* flag_new;         // [n_events]
    uint32_t* flag_rep;         // [n_events] then exclusive scan
    uint32_t* flag_front;       // [n_events] then exclusive scan
    uint32_t* scan_new;         // [n_events] exclusive scan of flag_new
    uint32_t state_base;
    uint32_t* new_state_event;  // [n_new] event of each new state
    uint32_t* next_frontier;
    uint32_t* level_max;        // [0..1] max ne, nocc of new states; [2..3] of the frontier;
                                // [4] largest match count of a (state, rule); [5] frontier
                                // states for the warp path
    // branchial
    uint32_t* bcount;           // [n_events] pairs (a, later b) per event a
    uint32_t* boff;             // [n_events+1] exclusive scan of bcount
    uint32_t* bpairs;           // output pairs (a, b)
    uint32_t bbase;             // pair index base
};

// Per-warp shared-memory carve-up, sized on the host from the level's largest state.
struct Layout {
    uint32_t NE, NOCC, CNE, CNOCC, V, W, NBR;
    uint32_t NV;        // distinct vertices a staged state may have (V = NV + fresh variables)
    uint32_t o_cur, o_nxt, o_csum, o_ccnt, o_nbr;                  // u64
    uint32_t o_peid, o_occ, o_ooff, o_nbo, o_deg, o_nn, o_comp;     // u32
    uint32_t o_cand, o_taken, o_misc;                               // u32
    uint32_t o_pevo, o_vloc, o_cvo, o_bind, o_match, o_mdepth;      // u16
    uint32_t o_pear, o_car;                                         // u8
    uint32_t o_rule;                                                // DevRule
    // lane-per-child path: parent occurrence and neighbour lists by vertex, per-vertex degree /
    // neighbour counts, and a batch of up to 32 matches (removed positions + produced local
    // vertices)
    uint32_t o_poff, o_pocc, o_pdeg, o_pnn, o_pnoff, o_pnbr, o_batch, o_mlist;
    uint32_t MCAP;      // matches the lane walk stages per (state, rule) (<= kLaneJoinCap)
    uint32_t region_bytes;   // lane layout without the trailing batch and match list (a warp's
                             // further parent regions need no batch or match list of their own)
    uint32_t o_pconn;   // u32: bit 0 = the parent is connected; bits 8.. = the arity every
                        // parent edge has when it is 2..4 (else 0)
    uint32_t o_pcnt;    // u32 per parent vertex: occurrences at position q in byte q (positions
                        // 0..3; filled when the parent's edges have one arity)
    // match forwarding: seeded schedule, creating event's consumed edges, delta matches (and a
    // sorted copy), a 32-match chunk of forwarded matches
    uint32_t o_sched2, o_fkc, o_dkey, o_dpos, o_dkey2, o_dpos2, o_fkey, o_fpos;
    uint32_t SB;                                                    // bytes per batch slot
    uint32_t VT, o_vtab, o_vtid;   // vertex hash table for large states (VT slots, 0 = unused)
    uint32_t o_srt;                // warp WL: sort buffer of the distinct-colour count
    // join indices of a staged state past kJoinIndexMin edges (XI = 1; count and warp layouts):
    // vertex -> state positions of the edges holding it (CSR), and the edges bucketed by
    // signature (at most kSigBuckets buckets); o_xready: bit 0 vertex index, bit 1 signature index
    uint32_t XI, o_xready, o_xoff, o_xinc, o_bkey, o_boff, o_blist;
    uint32_t bytes;
};

}  // namespace hgx
