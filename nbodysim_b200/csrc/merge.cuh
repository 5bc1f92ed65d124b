// Particle merging (merge.cu): the reference's minimum node size pass and its
// collision capture + merge, on the octree of the current step.
#pragma once

#include "common.cuh"

namespace nbody {

struct MergeBufs {
    uint32_t *label;   // user index -> representative user index (itself when not merged)
    uint32_t *rep;     // 1 at the representative of a merged group
    uint32_t *flag;    // collision endpoints / kept particles
    uint32_t *offs;    // exclusive scan of flag
    uint32_t *scan_tmp;
    double *mpos, *mvel, *mmass;  // merged values, stored at the representative
    double *pos2, *vel2, *mass2;  // compaction output
    void *acc2;
    uint64_t *skey_a, *skey_b;    // (component root) keys of the collision endpoints
    uint32_t *sidx_a, *sidx_b;
    uint32_t *sort_scratch;
    uint2 *pairs;
    uint32_t pair_cap;
    uint32_t *counters;  // kMc* below
};

enum : int {
    kMcPairs = 0,       // collision pairs found (may exceed pair_cap)
    kMcGroups = 1,      // minimum-size groups merged
    kMcKept = 2,        // particles left after compaction
    kMcInvolved = 3,    // particles that are endpoints of a collision pair
    kMcStatus = 4,      // kMergeStatus* bits
    kMcCount = 8,
};

enum : uint32_t {
    kMergeStatusUnion = 1u << 0,  // a union-find retry loop hit its bound (never expected)
    kMergeStatusTree = 1u << 1,   // a walk or fold met a malformed octree (never expected)
    kMergeStatusSort = 1u << 2,   // a radix-sort look-back gave up waiting (never expected)
};

// label[i] = i, rep[i] = 0, flag[i] = 0 for i < n; counters zeroed.
cudaError_t merge_begin(const MergeBufs &m, uint32_t n, cudaStream_t st, unsigned *launches);

// apply_minimum_size (src/main.cpp:1001-1060) on the built octree: every
// topmost cell whose side is below min_size and that holds >= 2 particles
// becomes one particle, folded in the reference's post-order child order.
cudaError_t merge_min_size(const MergeBufs &m, const Tree &t, const int32_t *oparent, const double *vel,
                           double min_size, cudaStream_t st, unsigned *launches);

// The collision capture of barnes_hut_thread (src/main.cpp:386-396): pairs
// (particle, accepted leaf) closer than `range`, found by a walk that replays
// the reference's opening decisions only where a leaf can be within range.
cudaError_t collide_find(const MergeBufs &m, const Tree &t, const int32_t *oparent, double theta, double range,
                         cudaStream_t st, unsigned *launches);
// Connected components of the pairs (root = smallest user index), endpoints
// scanned into a list; counters[kMcInvolved] = its length.
cudaError_t collide_components(const MergeBufs &m, uint32_t n, uint32_t npairs, cudaStream_t st, unsigned *launches);
// Orders the k endpoints by (component, user index) and folds each component
// with collide() (src/main.cpp:423-430) in that order.
cudaError_t collide_fold(const MergeBufs &m, uint32_t k, const double *pos, const double *vel, const double *mass,
                         cudaStream_t st, unsigned *launches);

// Keeps the particles whose label is themselves (merged values at the
// representatives, acceleration zero there, as a new particle has) and writes
// them, in user order, to pos2/vel2/mass2/acc2; counters[kMcKept] = count.
cudaError_t merge_compact(const MergeBufs &m, uint32_t n, const double *pos, const double *vel, const double *mass,
                          const void *acc, bool acc_double, cudaStream_t st, unsigned *launches);

}  // namespace nbody
