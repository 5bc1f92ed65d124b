/*
 * nbody_b200 -- an entry point that allocates nothing.
 *
 * No counterpart in the reference: fosted3/nbodysim always allocates its own
 * device buffers (src/cuda_code.cu:138-208). This entry point is for callers
 * that cannot call cudaMalloc -- code running while a stream is captured into
 * a CUDA graph, plug-ins whose host framework owns all device memory, and
 * loops that must never wait on an allocator. It computes the reference's root
 * cube (src/main.cpp:889-920: bounding-box midpoint, side = largest extent + 2,
 * a tie for the largest extent falling through to z) over particle arrays the
 * caller already holds in device memory. Its scratch lives in a fixed array
 * inside the library, held by every GPU context that loads the library until
 * that context ends.
 */
#ifndef NBODY_B200_NOALLOC_H
#define NBODY_B200_NOALLOC_H

#include <stdint.h>

#include "nbody_b200.h" /* status codes NBODY_OK, NBODY_ERR_* */

#ifdef __cplusplus
extern "C" {
#endif

/* Largest n accepted by nbody_root_cube_noalloc (4,194,304). */
uint32_t nbody_root_cube_noalloc_max_n(void);

/* d_pos: device array of n x 3 doubles (x, y, z per particle); d_mass: n
 * doubles on the device. Writes five doubles to the device array d_out:
 * center x, y, z, side, and a flag:
 *   0.0  the cube is valid;
 *   1.0  a position or mass is NaN or infinite: center and side are NaN;
 *   2.0  the library's scratch address did not belong to the running context
 *        (never expected; nothing was computed, center and side are NaN).
 * Work is queued on `stream` (a cudaStream_t, may be NULL); the call does not
 * wait for it.
 * Returns NBODY_ERR_INVALID for n == 0, n > nbody_root_cube_noalloc_max_n() or
 * a null pointer, before touching the GPU; NBODY_ERR_CUDA if the scratch
 * address cannot be looked up or the launch fails.
 * Set-up: the first call in each CUDA context looks up the device address of
 * the library's scratch array in that context, keyed by the context's unique
 * id. That includes the first call after cudaDeviceReset (a new primary
 * context) and the first call in a context created with the driver API. Make
 * that first call before any stream capture begins in the context.
 * Sharing: the scratch is shared by every call in a context and keeps the last
 * call's partial results; its completion ticket is back at zero when a call
 * finishes. Calls that overlap on the GPU race and must be serialised by the
 * caller. No cudaMalloc, cudaFree, cudaMemset or allocating library routine
 * is used. */
int nbody_root_cube_noalloc(const double *d_pos, const double *d_mass, uint32_t n, double *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
