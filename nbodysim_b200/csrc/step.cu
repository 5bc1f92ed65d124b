// Integration step, adaptive dt and FP64 diagnostics.
#include "step.cuh"

#include <algorithm>

namespace nbody {

// Semi-implicit Euler exactly as particle::update (src/particle.cpp:66-74):
// v = v + (a dt); x = x + (v dt), each product and sum rounded on its own.
// Adaptive dt (README.md:54-60 names the keys; the reference has no code):
//   dt_k = clamp(min(dt, max_vel_change / max|a|, max_pos_change / max|v|),
//                min_adaptive_dt, dt)
// with clamp as src/main.cpp:177-182 defines it and |v| taken before the kick.
// The FLOAT build (single) does the same in float: the state and dt are read
// as floats and every product and sum is rounded to float.
template <typename AccT>
__global__ void k_update(double *__restrict__ pos, double *__restrict__ vel, const AccT *__restrict__ acc,
                         uint32_t n, StepParams sp, DevScalars *sc) {
    griddep();
    double dt = sp.dt;
    if (sp.adaptive) {
        const double amax = __longlong_as_double((long long)sc->max_acc_bits);
        const double vmax = __longlong_as_double((long long)sc->max_vel_bits);
        double c = sp.dt;
        if (amax > 0.0) c = fmin(c, sp.max_vel_change / amax);
        if (vmax > 0.0) c = fmin(c, sp.max_pos_change / vmax);
        if (c < sp.min_adaptive_dt) c = sp.min_adaptive_dt;
        else if (c > sp.dt) c = sp.dt;
        dt = c;
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) sc->dt_used = dt;
    if (i >= n) return;
    if (sp.single) {
        const float fdt = __double2float_rn(dt);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t o = 3 * (size_t)i + k;
            const float v = __fadd_rn(__double2float_rn(vel[o]), __fmul_rn(__double2float_rn((double)acc[o]), fdt));
            vel[o] = (double)v;
            pos[o] = (double)__fadd_rn(__double2float_rn(pos[o]), __fmul_rn(v, fdt));
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const size_t o = 3 * (size_t)i + k;
        const double v = __dadd_rn(vel[o], __dmul_rn((double)acc[o], dt));
        vel[o] = v;
        pos[o] = __dadd_rn(pos[o], __dmul_rn(v, dt));
    }
}

// FP64 sums: kinetic, potential (1/2 sum m phi), momentum, angular momentum,
// mass, mass-weighted position. Block partials, then the last block sums the
// partials in block order, so the result does not depend on scheduling.
__global__ void k_diag(const double *__restrict__ pos, const double *__restrict__ vel,
                       const double *__restrict__ mass, const double *__restrict__ pot, uint32_t n,
                       double *__restrict__ partial, DevScalars *sc) {
    griddep();
    constexpr int K = kDiagCount;
    __shared__ double s_red[K][32];
    __shared__ bool s_last;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double m = mass[i];
        const double x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
        const double vx = vel[3 * (size_t)i], vy = vel[3 * (size_t)i + 1], vz = vel[3 * (size_t)i + 2];
        v[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        v[1] += pot ? 0.5 * m * pot[i] : 0.0;
        v[2] += m * vx; v[3] += m * vy; v[4] += m * vz;
        v[5] += m * (y * vz - z * vy);
        v[6] += m * (z * vx - x * vz);
        v[7] += m * (x * vy - y * vx);
        v[8] += m;
        v[9] += m * x; v[10] += m * y; v[11] += m * z;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double r = warp_sum(v[k]);
        if (lane == 0) s_red[k][wid] = r;
    }
    __syncthreads();
    if (wid == 0) {
        for (int k = 0; k < K; k++) {
            double r = lane < nw ? s_red[k][lane] : 0.0;
            r = warp_sum(r);
            if (lane == 0) partial[K * blockIdx.x + k] = r;
        }
        if (lane == 0) {
            __threadfence();
            s_last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    for (int k = 0; k < K; k++) {
        double acc = 0.0;
        for (uint32_t b = 0; b < gridDim.x; b++) acc += __ldcg(&partial[K * b + k]);
        sc->diag[k] = acc;
    }
    sc->ticket = 0;
}

__global__ void k_reset_pass(DevScalars *sc) {
    griddep();
    sc->interactions = 0;
    sc->walk_entries = 0;
    sc->walk_tiles = 0;
    sc->walk_decisions = 0;
    sc->walk_list = 0;
    sc->walk_near = 0;
    sc->n_onodes = 0;
    sc->depth = 0;
    sc->max_stack = 0;
    sc->fallback_tests = 0;
    sc->group_counter = 0;
    sc->ticket = 0;
    sc->deep_groups = 0;
    sc->word_ties = 0;
    sc->tie_runs = 0;
    sc->max_prefix_bits = 0;
    for (int k = 0; k < kPassBins; k++) sc->pair_passes[k] = 0;
    sc->max_acc_bits = 0;
    sc->max_vel_bits = 0;
}

__global__ void k_acc_to_double(const float *__restrict__ in, double *__restrict__ out, size_t count) {
    griddep();
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (double)in[i];
}

// ---- adjoint -----------------------------------------------------------------
// Reverse of particle::update (src/particle.cpp:66-74): with x' = x + v' dt and
// v' = v + a dt, the cotangents of step k follow from those of step k+1 as
//   mu = lv' + lx' dt;  lv = mu;  la = mu dt;  lx = lx' + (dF/dx)^T la.
__global__ void k_adj_pre(const double *__restrict__ lx, double *__restrict__ lv, double *__restrict__ lam, double dt,
                          uint32_t n) {
    griddep();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * (size_t)n) return;
    const double mu = lv[i] + lx[i] * dt;
    lv[i] = mu;
    lam[i] = mu * dt;
}

// Node cotangents -> particles. A particle j inside node n (its own leaf and
// every internal ancestor) receives (m_j / M_n) adj_c(n) in position, and
// (x_j - c_n) . adj_c(n) / M_n + adj_M(n) in mass, from c_n = sum m x / M_n.
template <typename GT>
__global__ void k_adj_distribute(const double4 *__restrict__ body, const uint32_t *__restrict__ sidx,
                                 const int32_t *__restrict__ leaf_oparent, const int32_t *__restrict__ oparent,
                                 const double4 *__restrict__ onode, const double *__restrict__ adj_node,
                                 const double *__restrict__ adj_leaf, const GT *__restrict__ gdir,
                                 const double *__restrict__ scale, double *__restrict__ lx, double *__restrict__ lm,
                                 uint32_t n) {
    griddep();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t ui = sidx[j];
    const double4 b = body[j];
    double gx = (double)gdir[3 * (size_t)ui], gy = (double)gdir[3 * (size_t)ui + 1], gz = (double)gdir[3 * (size_t)ui + 2];
    const double *al = adj_leaf + 4 * (size_t)j;
    gx += al[0]; gy += al[1]; gz += al[2];
    double gm = al[3];
    int p = n > 1 ? leaf_oparent[j] : -1;
    for (int hops = 0; p >= 0 && hops <= kMaxLevels + 1; hops++) {
        const double4 nd = onode[p];
        const double *an = adj_node + 4 * (size_t)p;
        if (nd.w != 0.0) {
            const double w = b.w / nd.w;
            gx += w * an[0]; gy += w * an[1]; gz += w * an[2];
            gm += ((b.x - nd.x) * an[0] + (b.y - nd.y) * an[1] + (b.z - nd.z) * an[2]) / nd.w;
        }
        gm += an[3];
        p = oparent[p];
    }
    if (scale) {  // the MIXED form's cotangents were scaled by a power of two
        const double f = *scale;
        gx *= f; gy *= f; gz *= f; gm *= f;
    }
    lx[3 * (size_t)ui] += gx; lx[3 * (size_t)ui + 1] += gy; lx[3 * (size_t)ui + 2] += gz;
    lm[ui] += gm;
}

cudaError_t launch_adj_pre(const double *lx, double *lv, double *lam, double dt, uint32_t n, cudaStream_t st) {
    const unsigned blocks = (unsigned)((3 * (size_t)n + 255) / 256);
    launch_pdl(k_adj_pre, dim3(blocks), dim3(256), 0, st, lx, lv, lam, dt, n);
    return cudaGetLastError();
}

cudaError_t launch_adj_distribute(const double4 *body, const uint32_t *sidx, const int32_t *leaf_oparent,
                                  const int32_t *oparent, const double4 *onode, const double *adj_node,
                                  const double *adj_leaf, const void *gdir, bool gdir_double, const double *scale,
                                  double *lx, double *lm, uint32_t n, cudaStream_t st) {
    const unsigned blocks = (n + 255) / 256;
    if (gdir_double)
        launch_pdl(k_adj_distribute<double>, dim3(blocks), dim3(256), 0, st, body, sidx, leaf_oparent, oparent, onode, adj_node, adj_leaf,
                                                         (const double *)gdir, scale, lx, lm, n);
    else
        launch_pdl(k_adj_distribute<float>, dim3(blocks), dim3(256), 0, st, body, sidx, leaf_oparent, oparent, onode, adj_node, adj_leaf,
                                                        (const float *)gdir, scale, lx, lm, n);
    return cudaGetLastError();
}

// Largest |v| over count doubles, into *out (ordered bits of a non-negative double).
__global__ void k_absmax(const double *__restrict__ v, size_t count, unsigned long long *out) {
    griddep();
    __shared__ double s_w[32];
    double m = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(v[i]));
    m = warp_max(m);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_w[w] = m;
    __syncthreads();
    if (w == 0) {
        m = lane < (int)(blockDim.x >> 5) ? s_w[lane] : 0.0;
        m = warp_max(m);
        if (lane == 0 && m > 0.0) atomic_max_nonneg(out, m);
    }
}

// out = in * 2^-e in FP32, where 2^e brings the largest |in| into [0.5, 1)
// (e = 0 when it is zero or not finite); sc->lam_scale = 2^e.
__global__ void k_scale_to_float(const double *__restrict__ in, float *__restrict__ out, size_t count,
                                 DevScalars *sc) {
    griddep();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double mx = __longlong_as_double((long long)sc->lam_max_bits);
    int e = 0;
    if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
    if (i == 0) sc->lam_scale = ldexp(1.0, e);
    if (i < count) out[i] = (float)ldexp(in[i], -e);
}

cudaError_t launch_lam_to_float_scaled(const double *in, float *out, size_t count, DevScalars *sc, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(&sc->lam_max_bits, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const size_t blocks = (count + 255) / 256;
    launch_pdl(k_absmax, dim3((unsigned)std::max<size_t>(1, std::min<size_t>(blocks, 1184))), dim3(256), 0, st, in, count,
                                                                                         &sc->lam_max_bits);
    launch_pdl(k_scale_to_float, dim3((unsigned)std::max<size_t>(1, blocks)), dim3(256), 0, st, in, out, count, sc);
    return cudaGetLastError();
}

cudaError_t launch_update(double *pos, double *vel, const void *acc, bool acc_double, uint32_t n,
                          const StepParams &sp, DevScalars *sc, cudaStream_t st) {
    const unsigned blocks = n ? (n + 255) / 256 : 1;
    if (acc_double)
        launch_pdl(k_update<double>, dim3(blocks), dim3(256), 0, st, pos, vel, (const double *)acc, n, sp, sc);
    else
        launch_pdl(k_update<float>, dim3(blocks), dim3(256), 0, st, pos, vel, (const float *)acc, n, sp, sc);
    return cudaGetLastError();
}

cudaError_t launch_diag(const double *pos, const double *vel, const double *mass, const double *pot,
                        uint32_t n, double *partial, unsigned blocks, DevScalars *sc, cudaStream_t st) {
    launch_pdl(k_diag, dim3(blocks), dim3(256), 0, st, pos, vel, mass, pot, n, partial, sc);
    return cudaGetLastError();
}

// max |a| and max |v| over n particles, recomputed into sc (adaptive dt when
// the walk's running maximum does not apply: after merging, or when the
// velocities arrive after the force pass).
template <typename AccT>
__global__ void k_maxima(const AccT *__restrict__ acc, const double *__restrict__ vel, uint32_t n, DevScalars *sc) {
    griddep();
    double amax = 0.0, vmax = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t o = 3 * (size_t)i;
        const double ax = acc[o], ay = acc[o + 1], az = acc[o + 2];
        const double vx = vel[o], vy = vel[o + 1], vz = vel[o + 2];
        amax = fmax(amax, sqrt(ax * ax + ay * ay + az * az));
        vmax = fmax(vmax, sqrt(vx * vx + vy * vy + vz * vz));
    }
    amax = warp_max(amax);
    vmax = warp_max(vmax);
    if ((threadIdx.x & 31) == 0) {
        atomic_max_nonneg(&sc->max_acc_bits, amax);
        atomic_max_nonneg(&sc->max_vel_bits, vmax);
    }
}

cudaError_t launch_maxima(const void *acc, bool acc_double, const double *vel, uint32_t n, DevScalars *sc,
                          cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(&sc->max_acc_bits, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->max_vel_bits, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess || n == 0) return e;
    const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 592);
    if (acc_double) launch_pdl(k_maxima<double>, dim3(blocks), dim3(256), 0, st, (const double *)acc, vel, n, sc);
    else launch_pdl(k_maxima<float>, dim3(blocks), dim3(256), 0, st, (const float *)acc, vel, n, sc);
    return cudaGetLastError();
}

cudaError_t launch_reset_pass(DevScalars *sc, cudaStream_t st) {
    launch_pdl(k_reset_pass, dim3(1), dim3(1), 0, st, sc);
    return cudaGetLastError();
}

cudaError_t launch_acc_to_double(const float *in, double *out, size_t count, cudaStream_t st) {
    if (!count) return cudaSuccess;
    launch_pdl(k_acc_to_double, dim3((unsigned)((count + 255) / 256)), dim3(256), 0, st, in, out, count);
    return cudaGetLastError();
}

}  // namespace nbody
