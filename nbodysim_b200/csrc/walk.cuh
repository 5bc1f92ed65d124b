// Fused tree walk + gravity (walk.cu).
#pragma once

#include "common.cuh"

namespace nbody {

constexpr int kWalkWarps = 4;       // warps per block
constexpr int kStackCap = 768;      // shared-memory stack entries per warp
constexpr int kSpillChunk = kStackCap / 2;
constexpr int kListFlush = 32;      // force pass once the interaction list holds this many
constexpr int kListCap = kListFlush + 32;

struct WalkArgs {
    Tree t;
    double theta;
    int damping;
    float *accf;        // MIXED: user order, 3 floats per particle
    double *accd;       // FP64: user order, 3 doubles per particle
    uint32_t *counts;   // optional: accepted nodes per particle (user order)
    double *pot;        // optional: potential phi_i per particle (user order)
    int2 *spill;        // per-warp spill regions (grid warps x spill_cap)
    uint32_t spill_cap;
    uint32_t n_groups;  // ceil(n / 32)
    int track_max_acc;  // reduce max |a| (adaptive dt)
};

// Launch shape of the persistent walk for this device (blocks to fill every SM).
struct WalkLaunch {
    unsigned blocks;
    size_t smem;
};
cudaError_t walk_launch_shape(bool fp64, int device, WalkLaunch *out);
cudaError_t launch_walk(const WalkArgs &a, bool fp64, const WalkLaunch &l, cudaStream_t st);

}  // namespace nbody
