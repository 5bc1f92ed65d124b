/*
 * Test infrastructure only: the oracle. Used by tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py as the CHECKER; never linked into the
 * product library.
 *
 * A plain-C restatement of fosted3/nbodysim's CPU hot path in the reference's
 * DOUBLE build, written to round exactly as the reference does so that results
 * are bit-identical to it (pinned by tests against oracle/_ref, which is the
 * reference's own code compiled unmodified):
 *   bho_generate     src/main.cpp:184-275 (std::default_random_engine draws)
 *   bho_build        src/main.cpp:887-927, src/octree.cpp:54-85, 134-196
 *   bho_mass_com     src/octree.cpp:203-221, 252-278
 *   bho_forces       src/main.cpp:306-333 (gravity), 335-421 (BFS walk)
 *   bho_update       src/particle.cpp:66-74, src/main.cpp:929-933
 * plus an FP64 direct-sum oracle (no reference counterpart). The _f32 entry
 * points restate the same path as the reference's FLOAT build (-DFLOAT, the
 * build its makefile ships) computes it, bit-identical to that build.
 * Arrays are AoS: pos[3*i+k], k = x,y,z.
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bho_gen_params {
    int gen_type;  /* 0 cube, 1 sphere, 2 shell */
    int mass_dist; /* 0 linear, 1 exp, 2 normal */
    int vel_dist;
    double size, min_mass, max_mass, min_vel, max_vel, r_sphere, rotation_magnitude;
    double rot_x, rot_y, rot_z, scale_x, scale_y, scale_z;
    unsigned long seed;
} bho_gen_params;

typedef struct bho_tree bho_tree;

/* Seeded initial conditions, bit-identical to the reference's DOUBLE build. */
int bho_generate(const bho_gen_params *g, uint32_t n, double *pos, double *vel, double *mass);

/* Root cube (src/main.cpp:898-920): center[3], side. */
void bho_root_cube(uint32_t n, const double *pos, double *center, double *side);

/* The same in the reference's FLOAT build (float extrema, float center and side). */
void bho_root_cube_f32(uint32_t n, const double *pos, double *center, double *side);

/* Pointer octree with one particle per leaf; NULL on allocation failure or when
 * two particles coincide (the reference recurses without bound there). */
bho_tree *bho_build(uint32_t n, const double *pos, const double *mass);
/* The same tree as the reference's FLOAT build makes it: positions and masses
 * rounded to float, child centres, masses and centres of mass in float
 * arithmetic; bho_forces on such a tree follows the FLOAT build's opening test
 * and gravity (results are floats widened to double). */
bho_tree *bho_build_f32(uint32_t n, const double *pos, const double *mass);
void bho_free(bho_tree *t);
int64_t bho_node_count(const bho_tree *t);
int bho_depth(const bho_tree *t);

/* Per-particle BFS walk + gravity (G = 6.67384e-11, no softening).
 * acc_out: n x 3. count_out (optional): accepted nodes per particle.
 * sample (optional): walk only those m particles (acc_out/count_out m long). */
int bho_forces(const bho_tree *t, double theta, int damping, int threads,
               const uint32_t *sample, uint32_t m, double *acc_out, uint32_t *count_out);

/* Semi-implicit Euler, in place: v += a dt; x += v dt. */
void bho_update(uint32_t n, double *pos, double *vel, const double *acc, double dt);

/* The FLOAT build's update (float arithmetic); pos/vel hold floats afterwards. */
void bho_update_f32(uint32_t n, double *pos, double *vel, const double *acc, double dt);

/* Full frames: build -> mass/COM -> walk -> update, `frames` times. */
int bho_run_frames(uint32_t n, double *pos, double *vel, const double *mass, double theta,
                   int damping, double dt, int threads, uint32_t frames, double *frames_out);
/* The same frame loop in the FLOAT build (float tree, walk, gravity and update). */
int bho_run_frames_f32(uint32_t n, double *pos, double *vel, const double *mass, double theta,
                       int damping, double dt, int threads, uint32_t frames, double *frames_out);

/* FP64 direct sum for the listed targets against all n sources (compensated
 * summation). acc_out: m x 3. */
int bho_direct(uint32_t n, const double *pos, const double *mass, int damping,
               const uint32_t *targets, uint32_t m, int threads, double *acc_out);

/* Branching nodes (>= 2 children) plus the root, pre-order; same record
 * layout as the reference harness's ref_tree_nodes. */
int bho_tree_nodes(const bho_tree *t, int cap, int *level, int *count, int *min_index,
                   double *node_mass, double *com, double *side);

#ifdef __cplusplus
}
#endif
#endif
