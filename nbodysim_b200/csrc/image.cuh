// Particle image rendering (image.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nbody {

struct ImageArgs {
    uint32_t w, h;
    int projection;  // 0 front, 1 side, 2 top, 3 iso
    int color;       // 0 bw, 1 heat
    int adaptive, nonlinear;
    double scale, brightness;
};

// grid: w*h doubles; maxbits: one u64; rgb: w*h*3 bytes (device). Asynchronous.
cudaError_t render_image(const double *pos, uint32_t n, const ImageArgs &a, double *grid,
                         unsigned long long *maxbits, uint8_t *rgb, cudaStream_t st);

}  // namespace nbody
