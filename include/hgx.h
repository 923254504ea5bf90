/*
 * hgx.h -- C ABI of the B200-native multiway evolution step.
 *
 * Plain pointers and sizes only; no C++ or torch types cross this boundary, and no exception
 * does either: every entry point returns an hgx_status, and hgx_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Each entry point names the reference interface it replaces (paths inside the reference
 * project). The evolution it computes is the reference engine's multiway step in WL mode:
 * states are identified by the shared WL canonical hash, events are every rule application
 * of every expanded state, causal edges are (producer, consumer, edge) triples, branchial
 * edges are event pairs of one input state that consumed a common edge.
 *
 * Blob encodings (uint32 arrays):
 *   rule   [n_lhs, (arity, var...)*n_lhs, n_rhs, (arity, var...)*n_rhs]   vars < 32, arity 1..16
 *   rules  [n_rules, rule...]
 *   roots  [n_roots, per root: n_edges, (arity, vertex...)*n_edges]
 *
 * Threading: one host thread drives one engine at a time; distinct engines are independent.
 */
#ifndef HGX_H
#define HGX_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HGX_API __attribute__((visibility("default")))
#else
#define HGX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hgx_status {
    HGX_OK = 0,
    HGX_ERR_INVALID = 1,    /* malformed rule / state / argument (reference: std::length_error,
                               std::invalid_argument from RuleBuilder and evolve) */
    HGX_ERR_CUDA = 2,       /* CUDA driver/runtime failure (reference: HG_CUDA_CHECK throw) */
    HGX_ERR_CAPACITY = 3,   /* a device capacity was exceeded (reference: ErrorKind overflow) */
    HGX_ERR_NO_DEVICE = 4,  /* no CUDA device: there is no CPU fallback */
    HGX_ERR_INTERNAL = 5
} hgx_status;

typedef struct hgx_engine hgx_engine;
typedef struct hgx_result hgx_result;

/* Options (hgx_engine_set_option). */
typedef enum hgx_option {
    /* ParallelEvolutionEngine::set_explore_from_canonical_states_only
       (hypergraph/include/hypergraph/parallel_evolution.hpp:926): 1 = expand each WL class
       once, at its shortest depth; 0 = full multiway (every raw state expanded). */
    HGX_OPT_QUOTIENT = 0,
    /* set_max_states (parallel_evolution.hpp:764): 0 = unlimited. */
    HGX_OPT_MAX_STATES = 1,
    /* set_transitive_reduction (parallel_evolution.hpp:781): 1 = the causal graph is reduced
       transitively (a (producer, consumer) pair implied by a longer path is dropped with all its
       triples), as hgcommon::tr_reduce. Evolutions of at most 64 levels; default 0. */
    HGX_OPT_TRANSITIVE_REDUCTION = 2,
    /* RecordSet::causal / ::branchial (common/include/hgcommon/core.hpp:128-155). */
    HGX_OPT_RECORD_CAUSAL = 3,
    HGX_OPT_RECORD_BRANCHIAL = 4,
    /* Read back every state's edge record (ids, arities, vertices); default 1. The reference
       returns state edge contents in every mode and adds the edge ids under
       EvolveInput::edge_identity (gpu/include/hg_gpu/evolve.hpp:36); the hg_gpu shim in
       hgx/compat.hpp keeps this on and selects the ids by edge_identity. */
    HGX_OPT_KEEP_STATE_EDGES = 5,
    /* 1 = record per-stage device times (CUDA events on the engine stream); 2 = time the expand
       kernel launches only (two events per launch; the other stages read 0). */
    HGX_OPT_TIMING = 6,
    /* 1 (default) = copy the result to host memory; 0 = keep it on the device and report the
       counts only (hgx_result_count works, hgx_result_copy returns empty arrays). */
    HGX_OPT_READBACK = 7,
    /* Incremental match forwarding (reference: ParallelEvolutionEngine::set_match_forwarding,
       parallel_evolution.hpp:775): a child's matches are its parent's matches that avoid the
       consumed edges plus the matches through the produced edges, instead of a full re-join.
       0 (default) = off, 1 = wherever it applies, 2 = states of 48 edges or more. Results are
       identical in every mode. */
    HGX_OPT_FORWARDING = 8,
    /* A level whose state caps (HGX_OPT_MAX_STATES / hgx_job.max_states) leave at least this many
       of its events past every cut is built in rounds that stop at each evolution's cut, so the
       dropped events are never built (default 8192; 0 = whenever a cap can cut). No reference
       counterpart; results are identical for every value. */
    HGX_OPT_CHUNK_MIN = 9,
    /* Event canonicalisation (Hypergraph::set_event_signature_keys, hypergraph.hpp:778;
       EvolveInput::event_canonicalization): hgcommon EventSignatureKeys bits over the WL
       canonical hashes -- 1 input state, 2 output state, 4 step, 8 rule (3 = the reference's
       Full preset). Events with equal signatures are one canonical event (HGX_COUNT_CANONICAL_EVENTS,
       HGX_ARR_EVENT_SIG); causal and branchial edges stay over every application, as in the
       reference. The edge-rank keys (16, 32; the Automatic preset) need an exact canonical
       labelling of every state and are rejected. Default 0. */
    HGX_OPT_EVENT_SIGNATURE_KEYS = 10,
    /* Join of the small-state expand kernel: 0 (default) = chosen per level by the engine's
       autotuner (device time per child, per bucket of children per frontier state), 1 = warp join,
       2 = lane-parallel walk. No reference counterpart; results are identical. */
    HGX_OPT_LANE_JOIN = 11,
    /* A single evolution under a state cap: a level whose cut the previous level's ratios place
       early in its frontier is counted and expanded as a frontier prefix first, the rest only if
       the cap is not reached. 0 (default) = prefix sized by that estimate, 1 = never split,
       N >= 2 = a prefix of N frontier states whenever the frontier is larger (for tests). No
       reference counterpart; results are identical for every value. */
    HGX_OPT_LEVEL_SPLIT = 12,
    /* Ceiling on the device memory the engine's arrays may hold, in bytes (0 = none, the
       default). A growth past it fails the call with HGX_ERR_CAPACITY before allocating, instead
       of pushing the GPU to a real out-of-memory. Replaces EvolveInput::max_device_memory_bytes
       (gpu/include/hg_gpu/evolve.hpp:136-141), whose one-shot evolve stops at the limit with a
       kDeviceOutOfMemory warning; the hg_gpu shim maps the error to that warning. */
    HGX_OPT_MAX_DEVICE_BYTES = 13,
    /* Join indices for staged states of more than 96 edges: 1 (default) = candidates for a
       pattern edge come from the bound vertex of smallest degree (the reference's
       InvertedVertexIndex, hypergraph/include/hypergraph/index.hpp:134-230) or, with no bound
       variable, from the signature buckets it is compatible with (SignatureIndex, index.hpp:30-130;
       common/include/hgcommon/signature_core.hpp:24-84); 0 = every edge is tested. Results are
       identical. */
    HGX_OPT_JOIN_INDEX = 14,
    /* With HGX_OPT_KEEP_STATE_EDGES: 1 (default) = the state records carry their global edge
       ids (HGX_ARR_STATE_EDGE_IDS); 0 = arities and vertices only, HGX_ARR_STATE_EDGE_IDS empty.
       The reference's results carry the ids only under EvolveInput::edge_identity
       (gpu/include/hg_gpu/evolve.hpp:36, default false); the hg_gpu shim maps it here. */
    HGX_OPT_KEEP_STATE_EDGE_IDS = 15,
    /* Result of a single evolution (hgx_evolve with readback): 1 (default) = when the engine's
       previous result was at least 64 MB, each finished frontier range's share of the result
       arrays is finalised and copied to the host while the later ranges compute (the copies
       overlap the evolution; page-locked blocks are sized from that previous result, and a result
       that outgrows them is copied whole at the end); 2 = the same for results of any size; 0 =
       the whole result is copied after the last level. Identical results. The reference reads its result back after the last step (gpu/src/evolve.cu:489-496). */
    HGX_OPT_STREAM_RESULT = 16
} hgx_option;

/* One evolution of a batch or a served request. */
typedef struct hgx_job {
    const uint32_t* rules;     /* rules blob */
    size_t rules_len;
    const uint32_t* roots;     /* roots blob */
    size_t roots_len;
    uint32_t steps;
    uint32_t quotient;         /* as HGX_OPT_QUOTIENT */
    uint64_t max_states;       /* as HGX_OPT_MAX_STATES */
} hgx_job;

/* Counts (hgx_result_count). */
typedef enum hgx_count {
    HGX_COUNT_STATES = 0,        /* states recorded: raw states (full) / class reps (quotient) */
    HGX_COUNT_EVENTS = 1,        /* Hypergraph::num_events (hypergraph.hpp:749) */
    HGX_COUNT_CLASSES = 2,       /* distinct WL canonical hashes (num_canonical_states, :694) */
    HGX_COUNT_CAUSAL = 3,        /* causal triples (CausalGraph::get_causal_edges) */
    HGX_COUNT_BRANCHIAL = 4,     /* branchial pairs (CausalGraph::get_branchial_edges) */
    HGX_COUNT_TRUNCATED = 5,     /* 1 when a state cap stopped the evolution */
    HGX_COUNT_CONSUMED = 6,      /* total consumed-edge entries over all events */
    HGX_COUNT_STATE_EDGES = 7,   /* total edge entries over all state records */
    HGX_COUNT_STATE_VERTS = 8,   /* total vertex entries over all state records */
    HGX_COUNT_RAW_STATES = 9,    /* Hypergraph::num_states (hypergraph.hpp:567): roots + events */
    HGX_COUNT_CANONICAL_EVENTS = 10 /* distinct event signatures under HGX_OPT_EVENT_SIGNATURE_KEYS
                                       (Hypergraph::num_events with event canonicalisation on,
                                       hypergraph.cpp:1639-1644); = EVENTS when off */
} hgx_count;

/* Arrays (hgx_result_copy); element type and length in brackets. */
typedef enum hgx_array {
    HGX_ARR_STATE_HASH = 0,      /* [u64 x STATES] WL canonical hash (CanonicalState::canonical_hash) */
    HGX_ARR_STATE_DEPTH = 1,     /* [u32 x STATES] */
    HGX_ARR_EVENTS = 2,          /* [u32 x EVENTS*4] (input state, output state, rule, step) */
    HGX_ARR_CAUSAL = 3,          /* [u32 x CAUSAL*3] (producer event, consumer event, edge) */
    HGX_ARR_BRANCHIAL = 4,       /* [u32 x BRANCHIAL*2] (event a, event b), a < b */
    HGX_ARR_EVENT_CONS_OFF = 5,  /* [u32 x EVENTS+1] */
    HGX_ARR_EVENT_CONS = 6,      /* [u32 x CONSUMED] consumed edge ids, pattern order */
    HGX_ARR_EVENT_PROD = 7,      /* [u32 x EVENTS*2] (first produced edge id, count) */
    HGX_ARR_STATE_EDGE_OFF = 8,  /* [u32 x STATES+1] (needs HGX_OPT_KEEP_STATE_EDGES) */
    HGX_ARR_STATE_EDGE_IDS = 9,  /* [u32 x STATE_EDGES] (empty under HGX_OPT_KEEP_STATE_EDGE_IDS = 0) */
    HGX_ARR_STATE_ARITY = 10,    /* [u8 x STATE_EDGES] (arity <= 16) */
    HGX_ARR_STATE_VERT_OFF = 11, /* [u32 x STATES+1] */
    HGX_ARR_STATE_VERTS = 12,    /* [u32 x STATE_VERTS] */
    HGX_ARR_EVENT_SIG = 13       /* [u64 x EVENTS] event signature (hg_gpu::Event::signature);
                                    empty unless HGX_OPT_EVENT_SIGNATURE_KEYS is set. The canonical
                                    event of a signature is its first event in this order. */
} hgx_array;

/* Message of the last failure on this thread ("" if none). */
HGX_API const char* hgx_last_error(void);

/* Library version string. */
HGX_API const char* hgx_version(void);

/* Replaces ParallelEvolutionEngine(Hypergraph*, num_threads)
   (hypergraph/include/hypergraph/parallel_evolution.hpp:743) and
   hg_gpu::Engine(EngineConfig) / PersistentEvolver (gpu/include/hg_gpu/evolve.hpp:435, :466):
   device state that persists across evolve calls. */
HGX_API hgx_status hgx_engine_create(int device, hgx_engine** out);
HGX_API void hgx_engine_destroy(hgx_engine* engine);

/* Replaces make_rule(i).lhs(...).rhs(...).build() (hypergraph/include/hypergraph/pattern.hpp:213)
   followed by ParallelEvolutionEngine::add_rule (parallel_evolution.hpp:756). */
HGX_API hgx_status hgx_engine_add_rule(hgx_engine* engine, const uint32_t* rule, size_t len);
HGX_API hgx_status hgx_engine_clear_rules(hgx_engine* engine);

/* Replaces the ParallelEvolutionEngine setters named on each hgx_option. */
HGX_API hgx_status hgx_engine_set_option(hgx_engine* engine, hgx_option opt, uint64_t value);

/* Replaces ParallelEvolutionEngine::evolve(initial_edges, steps) and its multi-root overload
   (parallel_evolution.hpp:1009, :1041), and hg_gpu::evolve(EvolveInput) (evolve.hpp:368). */
HGX_API hgx_status hgx_evolve(hgx_engine* engine, const uint32_t* roots, size_t roots_len, uint32_t steps,
                      hgx_result** out);

/* Many independent evolutions in one level-synchronous pipeline: one launch per stage per
   level for all of them. The batched form of hg_gpu::evolve (evolve.hpp:368); results are
   identical to evolving each job alone. out[i] receives job i's result. */
HGX_API hgx_status hgx_evolve_batch(hgx_engine* engine, const hgx_job* jobs, uint32_t n_jobs,
                            hgx_result** out);

/* Continuous batching. Replaces the strictly serial request loop of
   paclet_source/hg_evolve_main.cpp:99 (run_serve): requests are admitted between levels and
   advance together, each at its own depth. */
HGX_API hgx_status hgx_serve_reset(hgx_engine* engine);
HGX_API hgx_status hgx_serve_admit(hgx_engine* engine, const hgx_job* job, uint32_t* evolution_id);
/* Admit n jobs at once (one upload per array and one root-hashing launch for all of them);
   ids[i] receives job i's evolution id. Either every job is admitted or none is. */
HGX_API hgx_status hgx_serve_admit_batch(hgx_engine* engine, const hgx_job* jobs, uint32_t n,
                                         uint32_t* evolution_ids);
HGX_API hgx_status hgx_serve_step(hgx_engine* engine, int* still_active);
HGX_API hgx_status hgx_serve_take_finished(hgx_engine* engine, uint32_t* ids, uint32_t cap, uint32_t* n);
HGX_API hgx_status hgx_serve_collect(hgx_engine* engine, uint32_t evolution_id, hgx_result** out);
/* Collect n finished evolutions at once (one device finalisation and one copy for all of them). */
HGX_API hgx_status hgx_serve_collect_batch(hgx_engine* engine, const uint32_t* evolution_ids, uint32_t n,
                                           hgx_result** out);
HGX_API hgx_status hgx_serve_device_bytes(hgx_engine* engine, uint64_t* bytes);

/* Estimated device bytes one evolution will hold (state records, events, relations, dedup
   tables), from its rules, roots, step budget and state cap, without running it. Replaces
   hg_gpu::estimated_device_bytes(config_from_input(input)) (gpu/include/hg_gpu/evolve.hpp:404,
   :409); used by the serving loop's memory-budget admission. An uncapped evolution is
   estimated at the states its step budget can reach (bounded by 2^22). */
HGX_API hgx_status hgx_estimate_device_bytes(const hgx_job* job, uint64_t* bytes);

/* Free and total memory of a device (cudaMemGetInfo with that device current), for resolving
   EvolveInput::max_device_memory_bytes = 0 to 90% of the device's memory as the reference does
   (gpu/include/hg_gpu/evolve.hpp:136-141). */
HGX_API hgx_status hgx_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes);

/* Result accessors. Replace Hypergraph::num_states / num_events / num_canonical_states
   (hypergraph/include/hypergraph/hypergraph.hpp:567, :749, :694),
   CausalGraph::get_causal_edges / get_branchial_edges and the hg_gpu::EvolveResult vectors
   (gpu/include/hg_gpu/evolve.hpp:161-173). */
HGX_API uint64_t hgx_result_count(const hgx_result* result, hgx_count what);
HGX_API hgx_status hgx_result_copy(const hgx_result* result, hgx_array what, void* dst, size_t dst_bytes);
HGX_API void hgx_result_free(hgx_result* result);

/* Zero-copy access: *ptr points at the array inside the result (page-locked host memory for a
   single-evolution result), *count is its element count; valid until hgx_result_free. */
HGX_API hgx_status hgx_result_view(const hgx_result* result, hgx_array what, const void** ptr,
                                   uint64_t* count);
/* Every array at once: ptrs[a] / counts[a] for each hgx_array a (14 entries each), as
   hgx_result_view gives them one by one. */
HGX_API hgx_status hgx_result_views(const hgx_result* result, const void** ptrs, uint64_t* counts);

/* Device time per stage of the last evolve call, in milliseconds (HGX_OPT_TIMING must be on):
   out[0..7] = count, scan, expand, select, materialize, branchial, roots, total.
   launches: kernels launched by the call. */
HGX_API hgx_status hgx_engine_stage_times(hgx_engine* engine, double* out_ms, uint64_t* launches);

/* Counters of the last evolve call's expand kernels (the fused join + rewrite + WL + dedup
   kernels). out[0..4], lane-per-child kernel: bytes by the per-stage figures (join + rewrite +
   WL + dedup counted as separate HBM streams), bytes the fused kernel itself must move to or
   from HBM, children hashed, WL refinement rounds, launches. out[5..8], warp-per-child kernel:
   the same first four figures; out[9] its total device time in nanoseconds; out[10] lane-kernel
   launches that ran the lane-parallel walk (the join autotuner's choice; out has 11 entries). */
HGX_API hgx_status hgx_engine_expand_stats(hgx_engine* engine, uint64_t* out);

/* The last evolve call's result: out[0] = 1 if it was streamed (copied to the host range by
   range while the run continued, HGX_OPT_STREAM_RESULT), out[1] = the chunks copied. */
HGX_API hgx_status hgx_engine_result_stats(hgx_engine* engine, uint64_t* out);

/* The CUDA stream (cudaStream_t) the engine launches on, for callers that time or order
   work against it. */
HGX_API hgx_status hgx_engine_stream(hgx_engine* engine, void** stream);

/* Allocation-free WL hashing and deduplication of a batch of states that are already on the
   device. No counterpart in the reference: it exists for callers that cannot call cudaMalloc --
   code running under a runtime that owns the device's memory (a framework's caching allocator,
   a database or serving process with a fixed device budget) and code on a latency-critical path
   that cannot take cudaMalloc's implicit device synchronisation. It allocates nothing: the caller
   passes device buffers for the inputs and the outputs, and the scratch it needs (a dedup table
   of 2^20 slots, a work counter, an error word; about 12 MB) is a fixed array inside the library
   that every GPU which loads the library holds until the process exits.

   Inputs (device memory): states in the engine's record layout, concatenated in d_records; for
   state i, its record starts at word d_offsets[i] and holds d_num_edges[i] edge ids (any values;
   they only fix the edge order), then the edge arities packed four per 32-bit word (edge k in
   byte k % 4 of word k / 4), then the d_num_occ[i] vertex ids of the edges in order. max_edges /
   max_occ bound d_num_edges / d_num_occ and size the per-warp shared memory.
   Outputs (device memory): d_hash[i] = WL canonical hash of state i (bit-identical to the
   evolve path's state hashes); d_class[i] = the smallest index j with d_hash[j] == d_hash[i].

   At most 524,288 states per call (larger n_states is rejected with HGX_ERR_CAPACITY before any
   GPU work). The first call on a device resolves the array's device address (and sets the
   kernel's shared-memory limit) with that device current; make that first call before any stream
   capture. Every call clears and reuses the same array, so calls that overlap on the GPU (from
   two streams or two threads) race: serialise them. The call runs on `stream` (a cudaStream_t,
   NULL = legacy default stream) and synchronises it before returning, to report device-side
   errors as HGX_ERR_CAPACITY: a state larger than the declared bounds, or a record whose arities
   are outside 1..16 or do not add up to its d_num_occ entry (such a state is not hashed). The
   resolved address is kept for the life of the process: resetting the device (cudaDeviceReset)
   after the first call is not supported. */
HGX_API hgx_status hgx_hash_states_noalloc(const uint32_t* d_records, const uint64_t* d_offsets,
                                           const uint32_t* d_num_edges, const uint32_t* d_num_occ,
                                           uint32_t n_states, uint32_t max_edges, uint32_t max_occ,
                                           uint64_t* d_hash, uint32_t* d_class, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HGX_H */
