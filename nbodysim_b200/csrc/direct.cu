// FP64 direct-sum accelerations for error reports: every result of the
// Barnes-Hut path can be compared with the exact (all-pairs) sum on the same
// positions. One warp per target; each lane sums a stride of the sources with
// Neumaier compensation, and the 32 partial sums are combined in a fixed
// butterfly with exact two-sums, so the result does not depend on scheduling.
// The pair term follows gravity (src/main.cpp:306-333): normalize(d) * M * G * r^-2,
// or 1 / (r^2 + e^-r) with damping.
#include "direct.cuh"

namespace nbody {

namespace {

__device__ inline void neumaier(double &sum, double &comp, double g) {
    const double t = sum + g;
    comp += fabs(sum) >= fabs(g) ? (sum - t) + g : (g - t) + sum;
    sum = t;
}

// (s, c) += (s2, c2) with the rounding error of s + s2 kept exactly (TwoSum).
__device__ inline void combine(double &s, double &c, double s2, double c2) {
    const double t = s + s2;
    const double bp = t - s;
    const double err = (s - (t - bp)) + (s2 - bp);
    s = t;
    c = c + c2 + err;
}

__global__ void k_direct(const double *__restrict__ pos, const double *__restrict__ mass, uint32_t n, int damping,
                         const uint32_t *__restrict__ targets, uint32_t m, double *__restrict__ out) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m) return;
    const uint32_t i = targets ? targets[w] : w;
    const double xi = pos[3 * (size_t)i], yi = pos[3 * (size_t)i + 1], zi = pos[3 * (size_t)i + 2];
    double s[3] = {0.0, 0.0, 0.0}, c[3] = {0.0, 0.0, 0.0};
    for (uint32_t k = lane; k < n; k += 32) {
        if (k == i) continue;  // a particle exerts no force on itself
        const double dx = __dsub_rn(pos[3 * (size_t)k], xi), dy = __dsub_rn(pos[3 * (size_t)k + 1], yi),
                     dz = __dsub_rn(pos[3 * (size_t)k + 2], zi);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        const double r = __dsqrt_rn(r2);
        const double rs = damping ? 1.0 / (r2 + exp(-r)) : 1.0 / r2;
        const double f = __dmul_rn(__dmul_rn(mass[k], kG), rs);
        neumaier(s[0], c[0], __dmul_rn(__ddiv_rn(dx, r), f));
        neumaier(s[1], c[1], __dmul_rn(__ddiv_rn(dy, r), f));
        neumaier(s[2], c[2], __dmul_rn(__ddiv_rn(dz, r), f));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double s2 = __shfl_xor_sync(0xffffffffu, s[d], o);
            const double c2 = __shfl_xor_sync(0xffffffffu, c[d], o);
            // both partners combine in the same order (lower lane first) so they agree
            if (lane & o) {
                double a = s2, b = c2;
                combine(a, b, s[d], c[d]);
                s[d] = a; c[d] = b;
            } else {
                combine(s[d], c[d], s2, c2);
            }
        }
    }
    if (lane == 0) {
        out[3 * (size_t)w] = s[0] + c[0];
        out[3 * (size_t)w + 1] = s[1] + c[1];
        out[3 * (size_t)w + 2] = s[2] + c[2];
    }
}

}  // namespace

cudaError_t launch_direct(const double *pos, const double *mass, uint32_t n, int damping, const uint32_t *targets,
                          uint32_t m, double *out, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    const uint64_t threads = 32ull * m;
    k_direct<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(pos, mass, n, damping, targets, m, out);
    return cudaGetLastError();
}

}  // namespace nbody
