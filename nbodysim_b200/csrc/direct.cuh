// FP64 direct-sum accelerations (direct.cu).
#pragma once

#include "common.cuh"

namespace nbody {

// out[3w..3w+2] = the all-pairs FP64 acceleration of particle targets[w]
// (or w when targets is null), w < m. Asynchronous.
cudaError_t launch_direct(const double *pos, const double *mass, uint32_t n, int damping, const uint32_t *targets,
                          uint32_t m, double *out, cudaStream_t st);

}  // namespace nbody
