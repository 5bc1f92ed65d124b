// Particle image rendering on the GPU: the reference's write_image
// (src/main.cpp:556-678) as a scatter into an FP64 accumulation grid, a max
// reduction and a per-pixel tone map, producing the 24-bit bitmap the
// reference hands to FreeImage. Pixel (x, y) uses FreeImage's y (row 0 is the
// bottom row of the saved image).
#include "image.cuh"

namespace nbody {

namespace {

__device__ inline double clampd(double a, double x, double b) {  // src/main.cpp:177-182
    if (x < a) return a;
    if (x > b) return b;
    return x;
}

// Projection, scaling, bounds and clamping exactly as write_image computes
// them, every operation rounded on its own. Returns false for a particle the
// reference skips. `scale` is already doubled for the isometric view.
__device__ inline bool project(double px, double py, double pz, const ImageArgs &a, int *ix, int *iy) {
    const double hw = (double)(a.w / 2), hh = (double)(a.h / 2);  // integer halves, as the reference
    double x, y;
    switch (a.projection) {
        case 0: x = __dadd_rn(px, hw); y = __dadd_rn(pz, hh); break;  // front
        case 1: x = __dadd_rn(py, hw); y = __dadd_rn(pz, hh); break;  // side
        case 2: x = __dadd_rn(px, hw); y = __dadd_rn(py, hh); break;  // top
        default: {                                                     // iso
            const double s32 = __ddiv_rn(sqrt(3.0), 2.0);
            x = __ddiv_rn(__dadd_rn(__dmul_rn(s32, __dsub_rn(px, py)), (double)a.w), 2.0);
            const double sum = __dadd_rn(__dadd_rn(px, py), __dmul_rn(2.0, pz));
            y = __ddiv_rn(__dadd_rn(__dmul_rn(-0.5, sum), (double)a.h), 2.0);
        }
    }
    const double sm1 = __dsub_rn(a.scale, 1.0);
    x = __dadd_rn(x, __dmul_rn(__dsub_rn(x, hw), sm1));
    y = __dadd_rn(y, __dmul_rn(__dsub_rn(y, hh), sm1));
    // The reference bounds y by the width (src/main.cpp:603); kept as is.
    if (x < 0 || y < 0 || x > (double)(a.w - 1) || y > (double)(a.w - 1)) return false;
    x = clampd(0, x, (double)(a.w - 1));
    y = clampd(0, y, (double)(a.h - 1));
    if (a.projection == 3) y = __dsub_rn((double)(a.h - 1), y);
    *ix = (int)x;
    *iy = (int)y;
    return true;
}

__global__ void k_splat(const double *__restrict__ pos, uint32_t n, ImageArgs a, double *__restrict__ grid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ix, iy;
    if (project(pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], a, &ix, &iy))
        atomicAdd(&grid[(size_t)iy * a.w + ix], a.brightness);
}

__global__ void k_grid_max(const double *__restrict__ grid, size_t count, unsigned long long *maxbits) {
    double m = 0.0;  // the reference's max starts at 0
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, grid[i]);
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(m));
}

// (int) of a double the way x86 converts it: NaN and out-of-range give INT_MIN.
__device__ inline int to_int(double q) {
    if (!(q >= -2147483648.0 && q < 2147483648.0)) return (int)0x80000000u;
    return (int)q;
}

__global__ void k_tonemap(const double *__restrict__ grid, ImageArgs a, const unsigned long long *maxbits,
                          uint8_t *__restrict__ rgb) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)a.w * a.h) return;
    double mx = __longlong_as_double((long long)*maxbits);
    double t = grid[p];
    if (a.nonlinear) {
        mx = sqrt(mx);
        t = sqrt(t);
    }
    uint8_t r, g, b;
    if (a.color == 0) {  // BW
        const int v = a.adaptive ? to_int(clampd(0, __ddiv_rn(__dmul_rn(t, 255.0), mx), 255))
                                 : to_int(clampd(0, t, 255));
        r = g = b = (uint8_t)v;
    } else {  // HEAT
        int v = a.adaptive ? to_int(clampd(0, __ddiv_rn(__dmul_rn(t, 511.0), mx), 511)) : to_int(clampd(0, t, 511));
        if (v < 256) {
            b = (uint8_t)clampd(0, (double)(int)(255u - (unsigned)v), 255);
            g = (uint8_t)clampd(0, (double)v, 255);
            r = 0;
        } else {
            v -= 256;
            b = 0;
            g = (uint8_t)clampd(0, (double)(255 - v), 255);
            r = (uint8_t)clampd(0, (double)v, 255);
        }
    }
    rgb[3 * p] = r;
    rgb[3 * p + 1] = g;
    rgb[3 * p + 2] = b;
}

}  // namespace

cudaError_t render_image(const double *pos, uint32_t n, const ImageArgs &args, double *grid,
                         unsigned long long *maxbits, uint8_t *rgb, cudaStream_t st) {
    ImageArgs a = args;
    if (a.projection == 3) a.scale = a.scale * 2.0;  // src/main.cpp:577
    const size_t pixels = (size_t)a.w * a.h;
    cudaError_t e = cudaMemsetAsync(grid, 0, 8 * pixels, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (n) k_splat<<<(n + 255) / 256, 256, 0, st>>>(pos, n, a, grid);
    k_grid_max<<<296, 256, 0, st>>>(grid, pixels, maxbits);
    k_tonemap<<<(unsigned)((pixels + 255) / 256), 256, 0, st>>>(grid, a, maxbits, rgb);
    return cudaGetLastError();
}

}  // namespace nbody
