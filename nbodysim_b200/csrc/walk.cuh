// Fused tree walk + gravity (walk.cu).
#pragma once

#include "common.cuh"

namespace nbody {

constexpr int kWalkWarps = 4;       // default warps per block (the autotuner may pick 1 or 2)
constexpr int kWalkMaxWarps = 4;    // largest block the walk kernel is compiled for
constexpr int kStackCap = 640;      // shared-memory stack entries per warp
constexpr int kSpillChunk = kStackCap / 2;
// A tile pushes at most 32 lanes x 8 children; after a spill the stack must
// still have room for all of them.
static_assert(kStackCap - kSpillChunk >= 32 * 8, "a spill must leave room for one tile's pushes");
constexpr int kListFlush = 32;      // force pass once the interaction list holds this many
constexpr int kListCap = kListFlush + 32;

struct WalkArgs {
    Tree t;
    double theta;
    int damping;
    // The reference's FLOAT build: node values are floats and the opening test
    // is its float expression (float theta, float side / float distance).
    int single;
    float *accf;        // MIXED: user order, 3 floats per particle
    double *accd;       // FP64: user order, 3 doubles per particle
    uint32_t *counts;   // optional: accepted nodes per particle (user order)
    double *pot;        // optional: potential phi_i per particle (user order)
    int2 *spill;        // per-warp spill regions (grid warps x spill_cap)
    uint32_t spill_cap;
    uint32_t n_groups;  // ceil(n / 32)
    int track_max_acc;  // reduce max |a| (adaptive dt)
    int stats;          // collect the walk statistics (DevScalars walk_* and max_stack)
    // Adjoint mode (frozen decisions): the walk computes, for the cotangent
    // lam (dL/da per particle, user order), the direct term
    // gdir_i = -sum_n K_in lam_i and the node sums adj[n] = (sum_i K_in lam_i,
    // sum_i G g_in (d_in . lam_i)), internal nodes in adj_node, leaves (by
    // sorted index) in adj_leaf. K = dF/d(com) of the pair force.
    int adjoint;
    const float *lamf;  // MIXED
    const double *lamd; // FP64
    float *gdirf;       // MIXED: user order, 3 per particle
    double *gdird;      // FP64
    double *adj_node;   // 4 doubles per internal node
    double *adj_leaf;   // 4 doubles per sorted particle
    // Several independent systems: the work queue is a table of groups
    // (first sorted particle, count <= 32, system); each system has its own
    // octree root and root side. Null for a single system (groups of 32 from 0).
    const int4 *groups;
    const int32_t *sys_root_node;
    const double *sys_root;     // 4 per system: center xyz, side
};

// Launch shape of the persistent walk: `warps` per block, `blocks` in the grid
// (a whole number of resident blocks per SM), `smem` bytes per block.
struct WalkLaunch {
    unsigned blocks;
    unsigned warps;
    size_t smem;
};
// blocks_per_sm = 0: as many as fit. Returns the shape for that block size.
cudaError_t walk_launch_shape(bool fp64, int device, unsigned warps, unsigned blocks_per_sm, WalkLaunch *out);
// Resident blocks per SM that fit for `warps` per block (all walk variants).
cudaError_t walk_max_blocks_per_sm(bool fp64, unsigned warps, int *out);
cudaError_t launch_walk(const WalkArgs &a, bool fp64, const WalkLaunch &l, cudaStream_t st);

}  // namespace nbody
