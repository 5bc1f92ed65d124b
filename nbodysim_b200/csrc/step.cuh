// Integration, adaptive dt, diagnostics, small helpers (step.cu).
#pragma once

#include "common.cuh"

namespace nbody {

constexpr int kDiagCount = 12;

struct StepParams {
    double dt;
    int adaptive;
    double min_adaptive_dt, max_pos_change, max_vel_change;
    int single;  // the reference's FLOAT build: the update in float arithmetic
};

cudaError_t launch_update(double *pos, double *vel, const void *acc, bool acc_double, uint32_t n,
                          const StepParams &sp, DevScalars *sc, cudaStream_t st);
cudaError_t launch_diag(const double *pos, const double *vel, const double *mass, const double *pot,
                        uint32_t n, double *partial, unsigned blocks, DevScalars *sc, cudaStream_t st);
cudaError_t launch_reset_pass(DevScalars *sc, cudaStream_t st);
cudaError_t launch_maxima(const void *acc, bool acc_double, const double *vel, uint32_t n, DevScalars *sc,
                          cudaStream_t st);
cudaError_t launch_acc_to_double(const float *in, double *out, size_t count, cudaStream_t st);
// FP32 copy of count FP64 cotangents, scaled by the power of two that brings the
// largest into [0.5, 1) (the FP32 range would not hold them through many reverse
// steps); the factor back is left in sc->lam_scale.
cudaError_t launch_lam_to_float_scaled(const double *in, float *out, size_t count, DevScalars *sc, cudaStream_t st);
// mu = lv + lx dt -> lv; dL/da = mu dt -> lam (FP64)
cudaError_t launch_adj_pre(const double *lx, double *lv, double *lam, double dt, uint32_t n, cudaStream_t st);
cudaError_t launch_adj_distribute(const double4 *body, const uint32_t *sidx, const int32_t *leaf_oparent,
                                  const int32_t *oparent, const double4 *onode, const double *adj_node,
                                  const double *adj_leaf, const void *gdir, bool gdir_double, const double *scale,
                                  double *lx, double *lm, uint32_t n, cudaStream_t st);

}  // namespace nbody
