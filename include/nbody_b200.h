/*
 * nbody_b200 -- B200-native (sm_100a) Barnes-Hut engine: the C ABI.
 *
 * This library replaces the GPU force path of fosted3/nbodysim. The reference
 * exposes it as a C++ call,
 *     void barnes_hut_cuda(std::unordered_set<particle*>*, octree*, bool damping, datatype theta);
 *                                                            (src/cuda_helper.h:8)
 * backed by host-side tree walks and the chunk kernels behind run_compute
 * (src/cuda_code.h:6-21). Here the whole step -- root cube, octree build,
 * mass/centre-of-mass pass, per-particle walk + gravity, integration -- runs
 * on the GPU. Every entry point takes plain pointers and sizes and returns a
 * status code (0 = success) instead of exiting the process as the reference's
 * handle_error does (src/cuda_code.cu:29-37).
 *
 * Layouts. Host arrays are array-of-structs triples: pos[3*i + k], k = x, y, z,
 * in double precision (the reference's DOUBLE `datatype`, src/vector.h:4-13).
 * Particle i of every input keeps index i in every output.
 *
 * Semantics (identical to the reference's CPU path, src/main.cpp:335-421):
 *   root cube  = bbox midpoint, side = largest extent + 2 (ties: z extent)
 *   octree     = one particle per leaf, octant bits x=1, y=2, z=4, strict '>'
 *   open node  iff side / |com - x| > theta and the node is not a leaf
 *   accept     otherwise, unless the node is the particle's own leaf
 *   gravity    a += G M (com - x) / r^3, G = 6.67384e-11, no softening;
 *              damping: |a| = G M / (r^2 + e^-r)
 *   update     v += a dt; x += v dt
 *
 * Threading. A context belongs to one host thread at a time; all of its GPU
 * work is ordered on its own stream. Separate contexts may run concurrently.
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBODY_ABI_VERSION 7  /* 2: nbody_params.autotune, nbody_stats walk fields; 3: merging;
                                4: nbody_params.datatype_bytes; 5: nbody_stats sort fields;
                                6: nbody_stats.sort_tie_runs, nbody_set_walk_stats;
                                7: nbody_stats.sort_next_passes */

/* ---- status codes ---------------------------------------------------- */
#define NBODY_OK 0
#define NBODY_ERR_INVALID 1      /* bad argument (null pointer, n too large, theta <= 0 ...) */
#define NBODY_ERR_CUDA 2         /* a CUDA runtime call failed; see nbody_last_error_message */
#define NBODY_ERR_OOM 3          /* device or pinned-host allocation failed */
#define NBODY_ERR_COINCIDENT 4   /* two particles agree on all 63 octree levels; the reference
                                    recurses without bound on such input (src/octree.cpp:173-195) */
#define NBODY_ERR_NONFINITE 5    /* a position or mass is NaN or infinite */
#define NBODY_ERR_CAPACITY 6     /* a walk's node stack exceeded its spill capacity */
#define NBODY_ERR_NO_DEVICE 7    /* no CUDA device, or the device is not sm_100 */
#define NBODY_ERR_STATE 8        /* call out of order (e.g. step before particles are set) */

/* ---- configuration ---------------------------------------------------- */
#define NBODY_PRECISION_MIXED 0  /* FP32 pair forces + FP32 accumulation; FP64 tree, COM, state */
#define NBODY_PRECISION_FP64 1   /* the plain all-FP64 form of the same kernels */

typedef struct nbody_params {
    double theta;           /* opening angle, settings key `theta` (src/main.cpp:139) */
    double dt;              /* time step, key `dt` (src/main.cpp:140) */
    int damping;            /* key `damping` (src/main.cpp:127) */
    int adaptive;           /* key `adaptive` (README.md:54; no reference code) */
    double min_adaptive_dt; /* key `min_adaptive_dt` (README.md:56) */
    double max_pos_change;  /* key `max_pos_change` (README.md:58) */
    double max_vel_change;  /* key `max_vel_change` (README.md:60) */
    int precision;          /* NBODY_PRECISION_* */
    int device;             /* CUDA device ordinal */
    int autotune;           /* run nbody_autotune on the first step at each new size (default 0) */
    /* Merging, applied by nbody_step only (single system; not with the adjoint or
     * nbody_step_host, which keep n fixed). Each step may then shrink n; read it back
     * with nbody_device_view_get. */
    int collide;            /* key `collide` (src/main.cpp:130): merge particles closer than
                               collision_range that the walk accepts as leaves (src/main.cpp:386-396) */
    double collision_range; /* key `collision_range` (src/main.cpp:153, default 0.01) */
    double min_node_size;   /* key `min_node_size` (src/main.cpp:159): > 0 merges every cell
                               smaller than this into one particle before the forces
                               (apply_minimum_size, src/main.cpp:1001-1060) */
    int datatype_bytes;     /* the reference build whose decisions to reproduce: 8 = DOUBLE
                               (-DDOUBLE, default), 4 = FLOAT (-DFLOAT, the build its makefile
                               ships, makefile:3). With 4, positions, velocities and masses are
                               read as floats, and the root cube, child centres, node masses and
                               centres of mass, the opening test side/distance > theta and the
                               update are computed in float as that build computes them
                               (src/vector.h:4-13, src/octree.cpp:54-85, 203-313,
                               src/main.cpp:377, 887-927, src/particle.cpp:66-74), so accepted
                               nodes equal the FLOAT build's. Pair forces follow `precision`.
                               Merging and the adjoint need 8. */
} nbody_params;

/* Defaults of the reference's set_default (src/main.cpp:1312-1357) for the keys above;
 * adaptive-dt defaults from README.md:54-60; precision MIXED; device 0. */
void nbody_default_params(nbody_params *p);

typedef struct nbody_ctx nbody_ctx;

int nbody_create(const nbody_params *p, nbody_ctx **out);
int nbody_destroy(nbody_ctx *ctx);
int nbody_set_params(nbody_ctx *ctx, const nbody_params *p);
/* Optional: order this context's GPU work on a caller-owned cudaStream_t. */
int nbody_set_stream(nbody_ctx *ctx, void *cuda_stream);

/* ---- the drop-in force call -------------------------------------------
 * Replaces barnes_hut_cuda (src/cuda_helper.h:8, src/cuda_helper.cpp:218-246):
 * given n positions and masses (host memory), overwrite acc_out (host, n x 3)
 * with the Barnes-Hut acceleration of every particle. `damping` and `theta`
 * are the call's arguments exactly as in the reference signature; the
 * context's own values are not used. counts_out (optional, n) receives the
 * number of accepted nodes per particle. */
int nbody_barnes_hut(nbody_ctx *ctx, uint32_t n, const double *pos, const double *mass,
                     int damping, double theta, double *acc_out, uint32_t *counts_out);

/* ---- resident state ----------------------------------------------------
 * The frame loop of src/main.cpp:1420-1492 restricted to the hot path, with
 * the particle state kept in device memory between steps. */
int nbody_set_particles(nbody_ctx *ctx, uint32_t n, const double *pos, const double *vel,
                        const double *mass);
/* Declares the resident particles to be `nsys` independent systems stored one
 * after another, counts[s] particles each (every count >= 1). Each system gets
 * its own root cube and octree (as if it were its own reference run); one
 * persistent walk serves all systems from a shared work queue of 32-particle
 * groups. nsys = 1 restores a single system. nbody_barnes_hut always treats its
 * input as one system. (No reference counterpart: the reference runs one system.) */
int nbody_set_systems(nbody_ctx *ctx, uint32_t nsys, const uint32_t *counts);
/* Any output pointer may be NULL. acc is the last computed acceleration. */
int nbody_get_particles(nbody_ctx *ctx, double *pos, double *vel, double *acc);
/* Masses of the resident state (they change only by merging). */
int nbody_get_masses(nbody_ctx *ctx, double *mass);
/* nsteps full steps: root cube -> octree -> mass/COM -> walk+force -> (adaptive dt) -> update. */
int nbody_step(nbody_ctx *ctx, uint32_t nsteps);
/* Forces only, on the resident state (acc stays on the device). */
int nbody_compute_forces(nbody_ctx *ctx);
/* One step with host buffers in and out: upload pos/vel/mass, step, download pos/vel.
 * pos/vel are updated in place. From 65,536 particles the masses and velocities
 * are copied on a second stream while the first step's tree is built; with pinned
 * host buffers that copy overlaps the GPU work. */
int nbody_step_host(nbody_ctx *ctx, uint32_t n, double *pos, double *vel, const double *mass,
                    uint32_t nsteps);

/* Device addresses of the resident state (for zero-copy interop). Layout:
 * pos, vel: n x double3 (AoS); mass: n doubles; acc: n x float3 (MIXED) or
 * n x double3 (FP64). */
typedef struct nbody_device_view {
    uint32_t n;
    void *pos, *vel, *mass, *acc;
    int acc_is_double;
} nbody_device_view;
int nbody_device_view_get(nbody_ctx *ctx, nbody_device_view *out);

/* ---- statistics and diagnostics ---------------------------------------- */
typedef struct nbody_stats {
    uint64_t interactions;   /* accepted (particle, node) pairs in the last force pass */
    uint64_t interactions_total; /* summed over every pass of the last API call */
    uint64_t kernel_launches;    /* kernels this context has enqueued since creation */
    /* walk_entries .. walk_near and max_stack: collected only while
     * nbody_set_walk_stats(ctx, 1) is on (0 otherwise) */
    uint64_t walk_entries;       /* node entries tested by the walk's warps in the last pass */
    uint64_t walk_tiles;         /* stack tiles (<= 32 entries) the walk's warps staged */
    uint64_t walk_decisions;     /* internal nodes the warps decided (open / accept) */
    uint64_t walk_list;          /* bodies the warps put in their interaction lists */
    uint64_t walk_near;          /* bodies taken with FP64 offsets (too close for FP32 offsets) */
    uint32_t walk_warps_per_block; /* walk block shape in use (autotuned or default) */
    uint32_t walk_blocks;          /* walk grid size in use (persistent blocks) */
    uint32_t tree_nodes;     /* internal nodes of the (chain-free) octree */
    uint32_t tree_depth;     /* deepest internal-node level */
    uint32_t max_stack;      /* deepest walk stack seen (entries) */
    uint32_t fallback_tests; /* opening tests settled by the exact FP64 path */
    double last_dt;          /* dt used by the last step */
    double root_center[3];
    double root_side;
    float ms_tree, ms_com, ms_walk, ms_update; /* last pass, CUDA events; 0 if not timed */
    uint64_t merged_min_size;  /* particles removed by minimum-size merges in the last nbody_step */
    uint64_t merged_collisions; /* particles removed by collision merges in the last nbody_step */
    uint64_t collision_pairs;  /* (particle, leaf) pairs found within range, last nbody_step */
    uint32_t sort_passes;      /* 8-bit radix-sort passes of the last tree build: the planned ones,
                                  plus the full sort's 16 when the plan left a run of more than
                                  64 equal neighbours */
    uint32_t sort_split_bits;  /* key bits (3 per octree level) that separate every pair of
                                  Morton neighbours in the last build */
    uint32_t sort_tie_runs;    /* runs of neighbours equal over the planned bits (at most 64 each)
                                  that the last build sorted in place */
    uint32_t sort_next_passes; /* passes the next single step or force pass plans: the fewest that
                                  leave at most max(64, n / 16) pairs of the last build's neighbours
                                  tied (sorted in place as runs); for 8 calls after a build ran the
                                  full sort, the ones that cover sort_split_bits; 16 when a pair
                                  needs a third key word. A call of several steps plans the passes
                                  that cover sort_split_bits. A plan shrinks by two passes or more
                                  at a time. */
} nbody_stats;
int nbody_get_stats(nbody_ctx *ctx, nbody_stats *out);
/* Time phases with CUDA events on the context stream (default off; timed calls
 * launch kernels one by one). */
int nbody_set_timing(nbody_ctx *ctx, int enabled);
/* Collect the walk's statistics (nbody_stats walk_entries .. walk_near,
 * max_stack; default off). The forward walk then runs its counting instance,
 * a few % slower; forces and counts are the same either way. */
int nbody_set_walk_stats(nbody_ctx *ctx, int enabled);
/* Replay captured CUDA graphs for steps and adjoint steps (default on). Each
 * distinct configuration is captured on first use; a stream that cannot be
 * captured (the legacy default stream) falls back to direct launches. */
int nbody_set_graphs(nbody_ctx *ctx, int enabled);
/* Autotuner: times the walk on the resident state for each block shape (1, 2
 * or 4 warps per block, all or all-but-one resident blocks per SM) and keeps
 * the fastest for this context's precision (see nbody_stats.walk_*). */
int nbody_autotune(nbody_ctx *ctx);

typedef struct nbody_diagnostics {
    double kinetic;          /* sum 1/2 m v^2 */
    double potential;        /* 1/2 sum_i m_i phi_i over the Barnes-Hut walk */
    double momentum[3];      /* sum m v */
    double angular_momentum[3]; /* sum m x cross v */
    double mass;             /* total mass */
    double com[3];           /* centre of mass */
} nbody_diagnostics;
/* Energies and momenta of the resident state (FP64 reductions). Runs one
 * extra force pass with potentials. */
int nbody_get_diagnostics(nbody_ctx *ctx, nbody_diagnostics *out);

/* ---- differentiation ----------------------------------------------------
 * Reverse mode through the Barnes-Hut step with every step's opening decisions
 * and interaction lists frozen (no reference counterpart). Pair terms follow
 * the pair force's Jacobian; node terms flow through each node's centre of
 * mass and total mass to every particle inside it. In the MIXED form the
 * cotangents enter each FP32 pass scaled by a power of two that brings the
 * largest into [0.5, 1), and the FP64 results are scaled back, so gradients far
 * outside the FP32 range (they grow by many orders of magnitude through close
 * encounters) stay finite. */

/* Vector-Jacobian product of one force pass at the given state (host arrays):
 * dL_dpos = (da/dx)^T dL_dacc and dL_dmass = (da/dm)^T dL_dacc, n x 3 and n. */
int nbody_force_vjp(nbody_ctx *ctx, uint32_t n, const double *pos, const double *mass, const double *dL_dacc,
                    double *dL_dpos, double *dL_dmass);
/* nsteps fixed-dt steps from the resident state, keeping (pos, vel) every
 * `checkpoint_every` steps (0: ceil(sqrt(nsteps))). The state at nsteps stays
 * resident. Needs adaptive = 0. */
int nbody_forward_checkpointed(nbody_ctx *ctx, uint32_t nsteps, uint32_t checkpoint_every);
/* Reverse pass of the last nbody_forward_checkpointed: given dL/dpos and
 * dL/dvel at the final step (host n x 3; dL_dvel may be NULL for zero), writes
 * dL/dpos0, dL/dvel0 (n x 3) and dL/dmass (n) at the initial step. Segments
 * between checkpoints are recomputed forward, bit-identically. */
int nbody_backward(nbody_ctx *ctx, const double *dL_dpos, const double *dL_dvel, double *dL_dpos0,
                   double *dL_dvel0, double *dL_dmass);

/* ---- initial conditions ----------------------------------------------
 * Seeded generator of src/main.cpp:184-275 (std::default_random_engine, the
 * same draw order), so a seed gives the reference's particles bit for bit. */
typedef struct nbody_gen_params {
    int gen_type;    /* 0 cube, 1 sphere, 2 shell  (key gen_type) */
    int mass_dist;   /* 0 linear, 1 exp, 2 normal  (key mass_dist) */
    int vel_dist;    /* key vel_dist */
    double size, min_mass, max_mass, min_vel, max_vel, r_sphere, rotation_magnitude;
    double rotation_vector[3];
    double scale[3];
    uint64_t seed;
} nbody_gen_params;
void nbody_default_gen_params(nbody_gen_params *g);
int nbody_generate(const nbody_gen_params *g, uint32_t n, double *pos, double *vel, double *mass);

/* FP64 direct-sum (all-pairs) accelerations of the resident particles targets[0..m) (or of
 * particles 0..m-1 when targets is NULL), with the reference's pair term (src/main.cpp:306-333)
 * and compensated sums: the exact value that Barnes-Hut results are compared with. */
int nbody_direct_forces(nbody_ctx *ctx, uint32_t m, const uint32_t *targets, int damping, double *acc_out);

/* ---- frames and images -------------------------------------------------
 * The reference's frame files and renderer, on host arrays or the resident state. */

/* dir/NNNN.dat or dir/NNNN.txt (gen_filename, src/main.cpp:283-291; dir NULL: "./data"). */
int nbody_frame_path(const char *dir, uint32_t frame, int binary, char *buf, size_t buflen);
/* Binary frame (the resume format, src/main.cpp:730-743): per particle position, velocity,
 * acceleration (3 each) and mass in the reference's datatype (datatype_bytes 8 or 4).
 * acc may be NULL (written as zeros). */
int nbody_write_dat(const char *path, uint32_t n, const double *pos, const double *vel, const double *acc,
                    const double *mass, int datatype_bytes);
/* Reads a binary frame; with pos == NULL only sets *n. acc may be NULL. */
int nbody_read_dat(const char *path, int datatype_bytes, uint32_t *n, double *pos, double *vel, double *acc,
                   double *mass);
/* Text frame "x, y, z" per line, 6 significant digits (src/main.cpp:744-759). */
int nbody_write_txt(const char *path, uint32_t n, const double *pos, int datatype_bytes);
/* read_data's search (src/main.cpp:790-811): newest NNNN.dat <= num_frames in dir, or -1. */
int nbody_find_resume_frame(const char *dir, uint32_t num_frames, int32_t *frame_out);

/* The resident state as frame files dir/NNNN.dat (binary) and/or dir/NNNN.txt (text), the
 * records dump writes after each frame's update (src/main.cpp:680-766). Accelerations are
 * those of the last force pass (zeros before the first). */
int nbody_save_frame(nbody_ctx *ctx, const char *dir, uint32_t frame, int binary, int text, int datatype_bytes);
/* read_data (src/main.cpp:790-811): loads the newest dir/NNNN.dat <= num_frames into the
 * resident state and sets *next_frame to that frame + 1, or to 0 (state untouched) when
 * there is none. */
int nbody_load_frame(nbody_ctx *ctx, const char *dir, uint32_t num_frames, int datatype_bytes,
                     uint32_t *next_frame);

typedef struct nbody_image_params {
    uint32_t width, height; /* keys img_w, img_h */
    int projection;         /* key projection: 0 front, 1 side, 2 top, 3 iso */
    int color;              /* key color: 0 bw, 1 heat */
    int adaptive;           /* key adaptive_brightness */
    int nonlinear;          /* key nonlinear_brightness */
    double scale;           /* key scale */
    double brightness;      /* key brightness */
} nbody_image_params;
/* Defaults of set_default (src/main.cpp:1345-1352). */
void nbody_default_image_params(nbody_image_params *p);
/* write_image (src/main.cpp:556-678) on the GPU over the resident positions:
 * the 24-bit bitmap the reference passes to FreeImage, rgb_out[(y*width + x)*3 +
 * {R,G,B}], row y = 0 at the bottom of the image. With a fractional brightness the
 * per-pixel sums may round in a different order than the reference's. */
int nbody_render(nbody_ctx *ctx, const nbody_image_params *p, uint8_t *rgb_out);
/* Binary PPM of such a bitmap, top row first. */
int nbody_write_ppm(const char *path, uint32_t width, uint32_t height, const uint8_t *rgb);

/* ---- errors ------------------------------------------------------------ */
const char *nbody_status_string(int status);
/* Thread-local text of the last failure (CUDA error string or argument check). */
const char *nbody_last_error_message(void);

#ifdef __cplusplus
}
#endif
#endif /* NBODY_B200_H */
