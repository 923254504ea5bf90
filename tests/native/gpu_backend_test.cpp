// The worker's GPU backend (include/hgx/gpu_backend.hpp) on a named job; writes the WXF reply to
// argv[2]. Jobs: c1 (the triangle rule, 5 steps, full multiway, state mode Full), c1-genesis (the
// same with genesis events, global edges and state edge ids), c2q (C2's rule and initial state,
// 5 steps, quotient exploration, canonical hashes). Needs a GPU.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "hgx/gpu_backend.hpp"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: gpu_backend_test <job> <out.wxf>\n");
        return 2;
    }
    using Rules = std::vector<std::pair<std::string, std::vector<std::vector<std::vector<int64_t>>>>>;
    using States = std::vector<std::vector<std::vector<int64_t>>>;
    const std::string name = argv[1];
    Rules rules;
    States init;
    if (name.rfind("c1", 0) == 0) {
        rules = {{"r", {{{0, 1}, {1, 2}}, {{0, 1}, {1, 2}, {2, 0}}}}};
        init = {{{1, 2}, {2, 3}, {3, 1}}};
    } else {
        rules = {{"r", {{{0, 1}, {0, 2}}, {{0, 2}, {0, 3}, {1, 3}, {2, 3}}}}};
        init = {{{7, 7}, {7, 7}}};
    }
    hgx::compat::GpuJob job{rules, init};
    job.steps = 5;
    job.transitive_reduction = false;
    if (name == "c1-genesis") {
        job.show_genesis_events = true;
        job.include_global_edges = true;
        job.include_state_bitvectors = true;
    }
    if (name == "c2q") {
        job.steps = 5;
        job.explore_from_canonical_states_only = true;
        job.include_canonical_hashes = true;
        job.include_events_minimal = true;
    }
    hgx::compat::HostBridge host;
    std::vector<uint8_t> bytes;
    try {
        bytes = hgx::compat::run_gpu_evolution(job, host);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "run_gpu_evolution: %s\n", e.what());
        return 1;
    }
    std::ofstream(argv[2], std::ios::binary).write(reinterpret_cast<const char*>(bytes.data()),
                                                   static_cast<std::streamsize>(bytes.size()));
    std::printf("wrote %zu bytes\n", bytes.size());
    return 0;
}
