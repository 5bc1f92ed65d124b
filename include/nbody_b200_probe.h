/*
 * nbody_b200 -- measurement helper (no counterpart in the reference).
 *
 * The force kernel is bound by the FP32 CUDA-core pipe, whose peak is not in
 * the measured HBM / tensor-core peaks this project reports against. This
 * probe times a long chain of independent FP32 FMAs on every SM with CUDA
 * events and returns the achieved rate, the FP32 roofline denominator.
 */
#ifndef NBODY_B200_PROBE_H
#define NBODY_B200_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/* FP32 FMA throughput on `device`: *tflops = 2 * FMAs / time (TFLOP/s),
 * *ms = kernel time. Returns 0 on success (status codes of nbody_b200.h). */
int nbody_probe_fp32_peak(int device, double *tflops, double *ms);

#ifdef __cplusplus
}
#endif
#endif
