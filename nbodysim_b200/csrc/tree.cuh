// Octree construction: device buffers and the launch sequence (tree.cu).
#pragma once

#include "common.cuh"

namespace nbody {

struct TreeBuild {
    uint32_t n;
    const double *pos;          // user order, AoS
    const double *mass;
    cudaEvent_t mass_ready;     // non-null: the masses are still being copied on another stream;
                                // the build waits for this event before it first reads them
    const double *vel_for_max;  // non-null: also reduce max |v| (adaptive dt)
    int keep_root;              // rebuild inside the root cube already in sc (single system)
    // Sort plan (single system). sort_p2 passes sort the top 8 sort_p2 bits of
    // the second key word (levels 22-42; 0: none), then sort_p1 passes the top
    // 8 sort_p1 bits of the first word (levels 1-21); 8 passes take a whole
    // word. With sort_checked, runs of neighbours equal over those bits are
    // sorted in place by their full keys (sc->tie_runs), and the full two-word
    // sort runs on the device only when a run is longer than 64 (sc->word_ties),
    // so a plan that covers too few bits costs time, not results. The build
    // bins the pairs of neighbours by the passes that separate them
    // (sc->pair_passes) for the next plan. Several systems always take the full
    // sort.
    int sort_p1, sort_p2, sort_checked;
    cudaStream_t cond_stream;   // captures the full sort into a conditional graph node (used only
                                // while the build stream is being captured; null: never)
    unsigned *cond_launches;    // non-null: adds the kernels put in that conditional node (they
                                // run only when the planned sort left a long run)
    int single;                 // the reference's FLOAT build: positions and masses are read as
                                // floats; root cube, child centres, node masses and centres of
                                // mass are computed in float arithmetic
    DevScalars *sc;
    double *bbox_partial;       // 7 * bbox_blocks
    unsigned bbox_blocks;
    uint64_t *key_a, *key_b, *key2, *key3;
    uint32_t *idx_a, *idx_b;
    uint32_t *sort_scratch;     // sort_scratch_bytes(n)
    uint32_t *scan_tmp;         // ceil(max_len / 4096) + 1
    double4 *body;
    int32_t *bleft, *bright, *bparent, *leaf_bparent, *bdelta;
    uint32_t *head_flag, *head_id;
    int32_t *ochild, *ometa, *oparent, *leaf_oparent;
    uint32_t *ocount;
    double4 *onode;
    // Independent systems stored one after another (nsys > 1): each gets its
    // own root cube and octree; none of these is read when nsys == 1.
    uint32_t nsys;
    const uint32_t *sys_start;   // nsys + 1 offsets (user order)
    const uint32_t *sys_id;      // system of each particle (user order)
    uint32_t *sys_sorted;        // system of each sorted position
    double *sys_root;            // 4 doubles per system: center x, y, z, side
    int32_t *sys_root_node;      // octree root of each system (-1: fewer than 2 particles)
};

// Enqueues root cube -> keys -> sort -> bodies -> radix tree -> octree.
cudaError_t build_octree(const TreeBuild &tb, cudaStream_t st, unsigned *launches);
// Enqueues the bottom-up mass / centre-of-mass pass.
cudaError_t compute_com(const TreeBuild &tb, cudaStream_t st, unsigned *launches);

unsigned scan_exclusive(uint32_t *v, uint32_t len, uint32_t *tile_sums, uint32_t *total, cudaStream_t st);

}  // namespace nbody
