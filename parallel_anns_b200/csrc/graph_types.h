// Internal types shared by the graph construction units (graph_build.cu,
// nsg_build.cu) and the index code (panns_abi.cu).
#pragma once

#include <stdint.h>

#include <vector>

// A built graph in CSR form, returned through the opaque panns_graph handle
// of include/panns_build.h.
struct panns_graph {
    uint32_t n = 0, width = 0, entry = 0;
    std::vector<uint64_t> off;
    std::vector<uint32_t> nbrs;
    std::vector<uint32_t> knn;  // n x k (kept for the repair and for callers)
    uint32_t k = 0;
    uint32_t repaired = 0;
    // Cell-restricted construction only: each vertex's cell and each cell's
    // `probe` nearest cells (cells x probe).
    uint32_t cells = 0, probe = 0;
    std::vector<uint32_t> cell, near;
};

namespace panns {

// One output of glibc's rand() from the state panns_rand_seed set up
// (panns_abi.cu).
int32_t glibc_rand_next(int32_t *state);

}  // namespace panns
