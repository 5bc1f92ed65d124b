// Integration, adaptive dt, diagnostics, small helpers (step.cu).
#pragma once

#include "common.cuh"

namespace nbody {

constexpr int kDiagCount = 12;

struct StepParams {
    double dt;
    int adaptive;
    double min_adaptive_dt, max_pos_change, max_vel_change;
};

cudaError_t launch_update(double *pos, double *vel, const void *acc, bool acc_double, uint32_t n,
                          const StepParams &sp, DevScalars *sc, cudaStream_t st);
cudaError_t launch_diag(const double *pos, const double *vel, const double *mass, const double *pot,
                        uint32_t n, double *partial, unsigned blocks, DevScalars *sc, cudaStream_t st);
cudaError_t launch_reset_pass(DevScalars *sc, cudaStream_t st);
cudaError_t launch_acc_to_double(const float *in, double *out, size_t count, cudaStream_t st);

}  // namespace nbody
