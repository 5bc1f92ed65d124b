/*
 * Test infrastructure only. The reference's main.cpp calls barnes_hut_cuda
 * (declared at src/cuda_helper.h:8) when the `cuda` key is true. The CPU-only
 * oracle library never sets that key; this definition only satisfies the
 * linker and aborts loudly if it is ever reached.
 */
#include <cstdio>
#include <cstdlib>
#include "cuda_helper.h"

void barnes_hut_cuda(std::unordered_set<particle *> *, octree *, bool, datatype) {
    std::fprintf(stderr, "oracle: barnes_hut_cuda is not available in the CPU-only oracle build\n");
    std::abort();
}
