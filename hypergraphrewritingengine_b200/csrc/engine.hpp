// Host engine: device-resident multiway evolution over a batch of independent evolutions.
//
// This is the native runtime behind the C-ABI (include/hgx.h). It owns the device arrays,
// drives the level-synchronous step kernels and reads results back. One Engine serves the three
// ways the step is used:
//   * one evolution per call      (the plain path; what ParallelEvolutionEngine::evolve and
//                                  hg_gpu::evolve callers get)
//   * a batch of evolutions       (every level of every evolution in one launch per stage)
//   * a continuous request stream (admit between levels; finished evolutions are collected
//                                  while others keep running)
// No CPU fallback exists: without a CUDA device the constructor throws.
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace hgx {

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* expr, const char* file, int line)
        : std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(c) + " at " + file +
                             ":" + std::to_string(line) + " (" + expr + ")"),
          code(c) {}
};

// A rule as pattern-variable edge lists (variables < 32, arity 1..16, <= 16 edges per side).
struct RuleSpec {
    std::vector<std::vector<uint8_t>> lhs, rhs;
};

struct EvolutionSpec {
    std::vector<RuleSpec> rules;
    std::vector<std::vector<std::vector<uint32_t>>> roots;   // one or more initial states
    uint32_t steps = 0;
    bool quotient = true;        // true: each WL class expanded once, at its shortest depth
    uint64_t max_states = 0;     // 0 = unlimited; WL classes (quotient) or raw states (full)
};

// A result's arrays in one host block (page-locked when the block came from the device in a
// single copy), indexed like the C-ABI's hgx_array codes; `owner` frees the block.
struct ResultArrays {
    static constexpr int kArrays = 14;
    std::shared_ptr<void> owner;
    const void* ptr[kArrays] = {};
    uint64_t count[kArrays] = {};   // elements (u64 for the hashes, u32 otherwise)
};

struct EvolutionResult {
    // When set, the arrays live in `flat` (and the vectors below are empty).
    std::shared_ptr<ResultArrays> flat;
    uint64_t n_roots = 0;
    // States: in full multiway every raw state; in quotient mode one per WL class.
    std::vector<uint64_t> state_hash;
    std::vector<uint32_t> state_depth;
    std::vector<uint32_t> state_event;          // creating event (kNone for roots)
    std::vector<uint32_t> state_edge_off;       // [n+1] offsets into state_edge_ids (if kept)
    std::vector<uint32_t> state_edge_ids;
    std::vector<uint32_t> state_vert_off;       // [n+1] offsets into state_verts
    std::vector<uint8_t> state_arity;           // per edge, parallel to state_edge_ids
    std::vector<uint32_t> state_verts;
    // Events (ids local to this evolution, in canonical order).
    std::vector<uint32_t> ev_in, ev_out, ev_rule, ev_step;
    std::vector<uint32_t> ev_cons_off;          // [n+1]
    std::vector<uint32_t> ev_cons;              // consumed edge ids (pattern order)
    std::vector<uint32_t> ev_prod_first, ev_prod_count;
    // Relations over local event ids.
    std::vector<uint32_t> causal;               // (producer, consumer, edge) triples
    std::vector<uint32_t> branchial;            // (a, b) pairs, a < b
    std::vector<uint64_t> ev_sig;               // event signatures (event canonicalisation on)
    uint64_t num_classes = 0;
    uint64_t n_canonical_events = 0;            // distinct event signatures (= events when off)
    bool truncated = false;
    std::vector<std::string> warnings;
    // Set when the run kept its results on the device (RunOptions::readback == false): the
    // arrays above are empty and only these counts are filled.
    bool counts_only = false;
    uint64_t n_states = 0, n_events = 0, n_causal = 0, n_branchial = 0;
};

struct RunOptions {
    bool keep_state_edges = true;    // read back every state's edge record
    bool keep_state_edge_ids = true; // ... including its global edge ids (else arities, vertices)
    bool readback = true;            // false: leave results on the device, return counts
    bool causal = true;
    bool branchial = true;
    // Match forwarding: 0 = re-join every state, 1 = forward wherever it applies, 2 = forward
    // for states of 48 edges or more (results are identical in every mode).
    uint32_t forwarding = 0;
    // A level whose state caps leave at least this many events unneeded is expanded in rounds
    // that stop at each evolution's cut (results are identical either way).
    uint64_t chunk_min = 8192;
    // Transitive reduction of the causal graph (evolutions of at most 64 levels).
    bool transitive_reduction = false;
    // Event canonicalisation: hgcommon EventSignatureKeys bits 0-3 (input state, output state,
    // step, rule); 0 = every application is its own event.
    uint32_t event_keys = 0;
    // Join of the lane (small-state) expand kernel: 0 = autotuned per bucket of children per
    // frontier state, 1 = warp join, 2 = lane-parallel walk. Results are identical.
    uint32_t lane_join = 0;
    // Capped single evolution: 0 = split a level at the estimated cut, 1 = never, N >= 2 = at N.
    uint64_t level_split = 0;
    // Join indices (vertex and signature) for staged states past 96 edges: 1 = on, 0 = every
    // candidate is tested against every edge. Results are identical.
    uint32_t join_index = 1;
    // Single evolutions read back to the host: 1 = when the engine's last result was at least
    // 64 MB, each finished frontier range's share of the result is copied out while later ranges
    // compute (page-locked blocks sized from that result; one that outgrows them is copied whole
    // at the end); 2 = the same whatever the size; 0 = the whole result is copied at the end.
    // Identical results.
    uint32_t stream_result = 1;
};

// Per-stage device time of the last run (CUDA events on the engine stream), milliseconds.
struct StageTimes {
    double count = 0, scan = 0, expand = 0, expand_warp = 0, select = 0, materialize = 0,
           branchial = 0, roots = 0, total = 0;
    uint64_t launches = 0;   // kernels this engine launched during the run
    uint64_t expand_launches = 0;
    uint64_t walk_launches = 0;      // lane-kernel launches that used the lane-parallel walk
    uint64_t result_streamed = 0;    // 1: the result was copied out range by range during the run
    uint64_t result_chunks = 0;      // its chunks
    // lane-per-child expand kernel (k_expand<true>)
    uint64_t expand_bytes = 0;       // per-stage algorithmic bytes
    uint64_t expand_hbm_bytes = 0;   // bytes the fused kernel must move to/from HBM
    uint64_t children = 0;           // children built and WL-hashed
    uint64_t wl_rounds = 0;          // refinement rounds over all children
    // warp-per-child expand kernel (k_expand<false>), same four figures
    uint64_t warp_bytes = 0, warp_hbm_bytes = 0, warp_children = 0, warp_rounds = 0;
};

// Message returned by hgx_last_error() on the calling thread.
void set_last_error(const std::string& msg);

class Engine {
public:
    explicit Engine(int device = 0);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Run a batch of independent evolutions to completion; one result per spec.
    std::vector<EvolutionResult> run(const std::vector<EvolutionSpec>& specs,
                                     const RunOptions& opt = {});

    // Continuous-batching interface.
    void reset();                                   // drop everything, keep allocations
    uint32_t admit(const EvolutionSpec& spec);      // returns the evolution id (engine-wide)
    std::vector<uint32_t> admit(const std::vector<EvolutionSpec>& specs);   // all or none
    bool step(const RunOptions& opt = {});          // one level for every active evolution
    std::vector<uint32_t> take_finished();          // evolutions that completed since last call
    EvolutionResult collect(uint32_t evo, const RunOptions& opt = {});
    // several finished evolutions, finalised together (one set of launches and one copy)
    std::vector<EvolutionResult> collect(const std::vector<uint32_t>& evos, const RunOptions& opt = {});
    uint32_t active() const;
    uint64_t device_bytes_in_use() const;
    // Ceiling on the bytes the engine's device arrays may hold (0 = none): a growth past it
    // throws a capacity error instead of allocating (the call then fails with HGX_ERR_CAPACITY).
    void set_device_limit(uint64_t bytes);
    uint64_t device_limit() const;
    static uint64_t estimate_bytes(const EvolutionSpec& spec);

    cudaStream_t stream() const;
    void set_timing(int level);   // 0 off, 1 every stage, 2 the expand kernel only
    const StageTimes& times() const;
    void sync();

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace hgx
