// The C ABI (include/nbody_b200.h): contexts, device arena, pass sequencing.
//
// One pass over the hot path, all on the context's stream:
//   reset scalars -> root cube + keys + radix sort + octree (tree.cu)
//   -> bottom-up mass/COM (tree.cu) -> fused walk + gravity (walk.cu)
//   -> [update (step.cu)]
// The reference does the tree and the walk on the host and ships per-chunk
// interaction lists to the GPU every frame (src/cuda_helper.cpp:46-216); here
// nothing but the inputs and the results crosses PCIe, and device memory is a
// grow-only arena reused across calls (no per-call allocation after warm-up,
// in place of the reference's per-call cudaMalloc/cudaFree and cudaDeviceReset,
// src/cuda_code.cu:138-229).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>
#include <vector>

#include "../../include/nbody_b200.h"
#include "step.cuh"
#include "tree.cuh"
#include "sort.cuh"
#include "walk.cuh"
#include "image.cuh"
#include "merge.cuh"
#include "direct.cuh"

using namespace nbody;

namespace {

thread_local char g_msg[512] = "";

int fail(int code, const char *fmt, const char *detail = "") {
    std::snprintf(g_msg, sizeof g_msg, fmt, detail);
    return code;
}

#define NB_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            std::snprintf(g_msg, sizeof g_msg, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                          __FILE__, __LINE__);                                              \
            return e_ == cudaErrorMemoryAllocation ? NBODY_ERR_OOM : NBODY_ERR_CUDA;         \
        }                                                                                   \
    } while (0)

constexpr uint32_t kMaxParticles = 1u << 28;
constexpr uint32_t kSpillCap = 4096;  // entries per walk warp
constexpr unsigned kBboxBlocks = 592;
constexpr unsigned kDiagBlocks = 296;
constexpr uint32_t kOverlapMin = 65536;  // nbody_step_host overlaps the velocity upload from this size

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct nbody_ctx {
    nbody_params p;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t cap = 0, n = 0;
    bool have_state = false, have_vel = false, have_acc = false;
    // arena
    void *arena = nullptr;
    size_t arena_bytes = 0;
    double *pos = nullptr, *vel = nullptr, *mass = nullptr, *pot = nullptr, *acc_out = nullptr;
    void *acc = nullptr;  // float3 (MIXED) / double3 (FP64), user order
    uint32_t *counts = nullptr;
    TreeBuild tb{};
    double *diag_partial = nullptr;
    int2 *spill = nullptr;
    DevScalars *sc = nullptr;   // device
    DevScalars *hsc = nullptr;  // pinned mirror
    WalkLaunch wl_mixed{}, wl_fp64{};
    int timing = 0;
    int walk_stats = 0;  // nbody_set_walk_stats
    cudaEvent_t ev[5] = {};
    nbody_stats stats{};
    unsigned long long launches = 0;  // kernels enqueued by this context
    unsigned max_walk_warps = 0;      // spill regions allocated
    std::vector<unsigned char> tuned_key;  // configuration the autotuner last ran for
    // adjoint state (allocated on first use)
    void *adj_arena = nullptr;
    size_t adj_bytes = 0;
    double *lx = nullptr, *lv = nullptr, *lm = nullptr, *lam = nullptr, *gdir = nullptr;
    double *adj_node = nullptr, *adj_leaf = nullptr, *vel_work = nullptr, *seg_pos = nullptr, *ckpt = nullptr;
    // Octrees of one checkpoint segment, kept by the recomputation so that the
    // reverse pass at the same positions does not rebuild them (single system;
    // left out when the memory is not there).
    double *tree_slots = nullptr;
    uint32_t n_slots = 0;
    uint32_t fwd_steps = 0, fwd_every = 0, fwd_n = 0;
    double fwd_dt = 0.0;
    bool have_fwd = false;
    // independent systems (nbody_set_systems)
    uint32_t nsys = 1, sys_total = 0, ngroups = 0;
    void *sys_arena = nullptr;
    size_t sys_bytes = 0;
    uint32_t *sys_start = nullptr, *sys_id = nullptr, *sys_sorted = nullptr;
    int4 *groups = nullptr;
    double *sys_root = nullptr;
    int32_t *sys_root_node = nullptr;
    bool single_pass = false;  // nbody_barnes_hut: one system regardless of the layout
    // Sort plan of the next tree build (TreeBuild::sort_p1, sort_p2): the full
    // two-word sort until a build has measured its pairs of neighbours, then the
    // passes next_sort_plan picks from them. The build sorts the runs of
    // neighbours the plan leaves tied in place, and falls back to the full sort
    // on the device when a run is too long for that.
    int sort_p1 = 8, sort_p2 = 8;
    int sort_cooldown = 0;  // calls left whose plan follows the deepest split
    // Calls of several steps replay one captured step whose plan cannot change
    // while the state drifts: they sort by the deepest split (sort_deep_p1, p2).
    int sort_deep_p1 = 8, sort_deep_p2 = 8;
    bool multi_step_call = false;
    // CUDA graphs: one captured step replayed per step; per-offset graphs for the
    // adjoint's recompute and reverse steps. Rebuilt when their key changes.
    bool use_graphs = true;
    std::vector<unsigned char> step_key, adj_key;
    cudaGraphExec_t step_exec = nullptr;
    unsigned step_launches = 0;
    unsigned step_cond_launches = 0;  // of those, the kernels of the full sort's conditional node
    unsigned capture_cond_launches = 0;
    unsigned replayed_cond_launches = 0;  // of the last replayed step, added if its full sort ran
    std::vector<cudaGraphExec_t> rec_exec, adj_exec;
    std::vector<unsigned> rec_launches, adj_launches;
    // image rendering buffers (grown on demand)
    void *img_arena = nullptr;
    size_t img_bytes = 0;
    // merging (collisions, minimum node size): buffers sized for cap, pairs grown on demand
    void *merge_arena = nullptr;
    size_t merge_bytes = 0;
    uint32_t merge_cap = 0;
    MergeBufs mb{};
    uint2 *pairs = nullptr;
    uint32_t *hcounters = nullptr;  // pinned mirror of mb.counters
    uint64_t merged_min_size = 0, merged_collisions = 0, collision_pairs = 0;
    // nbody_direct_forces: targets and results (grown on demand)
    void *direct_arena = nullptr;
    size_t direct_bytes = 0;
    // nbody_step_host: masses and velocities uploaded on a second stream while the tree is built
    cudaStream_t aux_stream = nullptr;
    // captures the tree build's full sort into a conditional graph node
    cudaStream_t cond_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_mass = nullptr, ev_vel = nullptr;
    cudaEvent_t mass_pending = nullptr;  // set while a force pass must wait for ev_mass before reading masses
};

namespace {

// The reference's FLOAT build: decisions and node values follow its float arithmetic.
bool single(const nbody_ctx *c) { return c->p.datatype_bytes == 4; }

int set_device(nbody_ctx *c) {
    NB_CUDA(cudaSetDevice(c->p.device));
    return NBODY_OK;
}

int check_params(const nbody_params *p) {
    if (!p) return fail(NBODY_ERR_INVALID, "params is null%s");
    if (!(p->theta > 0.0) || !std::isfinite(p->theta)) return fail(NBODY_ERR_INVALID, "theta must be finite and > 0%s");
    if (!std::isfinite(p->dt)) return fail(NBODY_ERR_INVALID, "dt must be finite%s");
    if (p->precision != NBODY_PRECISION_MIXED && p->precision != NBODY_PRECISION_FP64)
        return fail(NBODY_ERR_INVALID, "unknown precision%s");
    if (p->adaptive && (!(p->max_pos_change > 0) || !(p->max_vel_change > 0) || !(p->min_adaptive_dt >= 0)))
        return fail(NBODY_ERR_INVALID, "adaptive dt needs max_pos_change > 0, max_vel_change > 0, min_adaptive_dt >= 0%s");
    if (!(p->collision_range >= 0) || !std::isfinite(p->collision_range))
        return fail(NBODY_ERR_INVALID, "collision_range must be finite and >= 0%s");
    if (!(p->min_node_size >= 0) || !std::isfinite(p->min_node_size))
        return fail(NBODY_ERR_INVALID, "min_node_size must be finite and >= 0%s");
    if (p->datatype_bytes != 8 && p->datatype_bytes != 4)
        return fail(NBODY_ERR_INVALID, "datatype_bytes must be 8 (DOUBLE build) or 4 (FLOAT build)%s");
    if (p->datatype_bytes == 4 && (p->collide || p->min_node_size > 0))
        return fail(NBODY_ERR_INVALID, "collisions and min_node_size need datatype_bytes 8%s");
    return NBODY_OK;
}

// Carves every per-particle buffer out of one allocation sized for `cap`.
int reserve(nbody_ctx *c, uint32_t n) {
    if (n <= c->cap && c->arena) return NBODY_OK;
    uint32_t cap = n < 1024 ? 1024 : n + n / 4;
    if (cap > kMaxParticles) cap = kMaxParticles;
    const size_t N = cap;
    const size_t sort_blocks = (N + 4095) / 4096;
    const size_t scan_tiles = (256 * sort_blocks + 4095) / 4096 + (N + 4095) / 4096 + 8;
    const size_t spill_entries = (size_t)c->max_walk_warps * kSpillCap;
    struct Piece { void **dst; size_t bytes; };
    TreeBuild &tb = c->tb;
    Piece pieces[] = {
        {(void **)&c->pos, 24 * N}, {(void **)&c->vel, 24 * N}, {(void **)&c->mass, 8 * N},
        {(void **)&c->acc, 24 * N}, {(void **)&c->acc_out, 24 * N}, {(void **)&c->counts, 4 * N},
        {(void **)&c->pot, 8 * N},
        {(void **)&tb.key_a, 8 * N}, {(void **)&tb.key_b, 8 * N}, {(void **)&tb.key2, 8 * N},
        {(void **)&tb.key3, 8 * N}, {(void **)&tb.idx_a, 4 * N}, {(void **)&tb.idx_b, 4 * N},
        {(void **)&tb.sort_scratch, sort_scratch_bytes(cap)}, {(void **)&tb.scan_tmp, 4 * scan_tiles},
        {(void **)&tb.body, 32 * N}, {(void **)&tb.onode, 32 * N},
        {(void **)&tb.bleft, 4 * N}, {(void **)&tb.bright, 4 * N}, {(void **)&tb.bparent, 4 * N},
        {(void **)&tb.leaf_bparent, 4 * N}, {(void **)&tb.bdelta, 4 * N},
        {(void **)&tb.head_flag, 4 * N}, {(void **)&tb.head_id, 4 * N}, {(void **)&tb.ocount, 4 * N},
        {(void **)&tb.ochild, 32 * N}, {(void **)&tb.ometa, 4 * N}, {(void **)&tb.oparent, 4 * N},
        {(void **)&tb.leaf_oparent, 4 * N},
        {(void **)&tb.bbox_partial, 8 * 7 * kBboxBlocks}, {(void **)&c->diag_partial, 8 * kDiagCount * kDiagBlocks},
        {(void **)&c->spill, 8 * spill_entries},
    };
    size_t total = 0;
    for (auto &pc : pieces) total += align256(pc.bytes);
    if (c->arena) {
        NB_CUDA(cudaStreamSynchronize(c->stream));
        NB_CUDA(cudaFree(c->arena));
        c->arena = nullptr;
        c->cap = 0;
    }
    void *arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(NBODY_ERR_OOM, "device arena allocation failed (%s)", cudaGetErrorString(e));
    }
    char *p = (char *)arena;
    for (auto &pc : pieces) {
        *pc.dst = p;
        p += align256(pc.bytes);
    }
    c->arena = arena;
    c->arena_bytes = total;
    c->cap = cap;
    tb.bbox_blocks = kBboxBlocks;
    tb.sc = c->sc;
    c->have_state = c->have_vel = c->have_acc = false;
    return NBODY_OK;
}

// The next build's sort plan, in whole 8-bit passes: the top bits of the first
// key word, or all of it and the top bits of the second. The deepest split of
// the last build (the key bits that separate every pair of neighbours) gives
// the plan that leaves no ties. A single step or force pass takes the fewest
// passes that leave at most max(64, n / kTieShare) pairs of neighbours tied,
// which the build sorts in place as short runs; after a build whose runs were
// too long for that (it ran the full sort), the deepest split sets that plan
// for kPlanCooldown calls. A call of several steps replays one captured step
// while the state drifts, and ties that grow past a run of 64 would make every
// later step run the full sort: it takes the deepest split (the 256-step
// forward of the adjoint's sphere of 65,536: 239 ms with the fewer passes, 180
// ms with the deepest split). A split beyond two key words keeps the full sort.
// A plan shrinks only by two passes or more, so that small changes do not
// rebuild captured graphs; it grows at once, and the deepest-split plan also
// follows a build that sorted runs or ran the full sort. No split measured:
// keep the plans.
constexpr uint32_t kTieShare = 16;
constexpr int kPlanCooldown = 8;

void next_sort_plan(nbody_ctx *c, const DevScalars &h) {
    if (h.max_prefix_bits == 0) return;
    const int deepest = std::min(passes_for_bits(h.max_prefix_bits), 16);
    if (h.word_ties) c->sort_cooldown = kPlanCooldown;
    int want = deepest;
    if (deepest < 16 && c->sort_cooldown == 0) {
        const uint64_t tol = std::max<uint64_t>(64, c->n / kTieShare);
        uint64_t tied = 0;  // pairs that a plan of want - 1 passes leaves tied
        while (want > 1) {
            tied += h.pair_passes[want];
            if (tied > tol) break;
            want--;
        }
    }
    if (c->sort_cooldown > 0) c->sort_cooldown--;
    const int p1 = std::min(want, 8), p2 = want - p1;
    const int cur = c->sort_p1 + c->sort_p2;
    if (h.word_ties || want > cur || cur - want >= 2) {
        c->sort_p1 = p1;
        c->sort_p2 = p2;
    }
    const int cur_deep = c->sort_deep_p1 + c->sort_deep_p2;
    if (h.word_ties || h.tie_runs || deepest > cur_deep || cur_deep - deepest >= 2) {
        c->sort_deep_p1 = std::min(deepest, 8);
        c->sort_deep_p2 = deepest - c->sort_deep_p1;
    }
}

// Marks an API call of several steps for its duration (tree_inputs picks the
// deepest-split sort plan).
struct MultiStepCall {
    nbody_ctx *c;
    bool saved;
    MultiStepCall(nbody_ctx *ctx, bool multi) : c(ctx), saved(ctx->multi_step_call) { c->multi_step_call = multi; }
    ~MultiStepCall() { c->multi_step_call = saved; }
};

int check_status(nbody_ctx *c) {
    NB_CUDA(cudaStreamSynchronize(c->stream));
    const DevScalars &h = *c->hsc;
    nbody_stats &s = c->stats;
    s.interactions = h.interactions;
    s.interactions_total = h.interactions_total;
    s.walk_entries = h.walk_entries;
    s.walk_tiles = h.walk_tiles;
    s.walk_decisions = h.walk_decisions;
    s.walk_list = h.walk_list;
    s.walk_near = h.walk_near;
    if (h.word_ties) c->launches += c->replayed_cond_launches;  // the replayed step ran its full sort
    c->replayed_cond_launches = 0;
    s.kernel_launches = c->launches;
    {
        const WalkLaunch &w = c->p.precision == NBODY_PRECISION_FP64 ? c->wl_fp64 : c->wl_mixed;
        s.walk_warps_per_block = w.warps;
        s.walk_blocks = w.blocks;
    }
    s.merged_min_size = c->merged_min_size;
    s.merged_collisions = c->merged_collisions;
    s.collision_pairs = c->collision_pairs;
    s.tree_nodes = h.n_onodes;
    s.tree_depth = h.depth;
    s.max_stack = h.max_stack;
    s.fallback_tests = h.fallback_tests;
    s.last_dt = h.dt_used;
    for (int k = 0; k < 3; k++) s.root_center[k] = h.root_center[k];
    s.root_side = h.root_side;
    const int used_plan = c->multi_step_call ? c->sort_deep_p1 + c->sort_deep_p2 : c->sort_p1 + c->sort_p2;
    s.sort_passes = c->nsys > 1 ? 18u : (uint32_t)used_plan + (h.word_ties ? 16u : 0u);
    s.sort_split_bits = h.max_prefix_bits;
    s.sort_tie_runs = h.tie_runs;
    next_sort_plan(c, h);
    s.sort_next_passes = c->nsys > 1 ? 18u : (uint32_t)(c->sort_p1 + c->sort_p2);
    if (c->timing) {
        float ms[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; k++) cudaEventElapsedTime(&ms[k], c->ev[k], c->ev[k + 1]);
        cudaGetLastError();  // an unrecorded event must not leak into later checks
        s.ms_tree = ms[0]; s.ms_com = ms[1]; s.ms_walk = ms[2]; s.ms_update = ms[3];
    }
    if (h.status & kStatusNonFinite) return fail(NBODY_ERR_NONFINITE, "a position or mass is NaN or infinite%s");
    if (h.status & kStatusCoincident)
        return fail(NBODY_ERR_COINCIDENT, "particles coincide to 63 octree levels (the reference recurses without bound)%s");
    if (h.status & kStatusCapacity) return fail(NBODY_ERR_CAPACITY, "walk stack spill capacity exceeded%s");
    if (h.status & kStatusSortStall) return fail(NBODY_ERR_CUDA, "radix sort look-back gave up waiting%s");
    return NBODY_OK;
}

void tree_inputs(nbody_ctx *c, uint32_t n, bool want_vmax) {
    TreeBuild &tb = c->tb;
    tb.n = n;
    tb.pos = c->pos;
    tb.mass = c->mass;
    tb.mass_ready = c->mass_pending;
    tb.vel_for_max = want_vmax ? c->vel : nullptr;
    tb.sc = c->sc;
    tb.single = single(c) ? 1 : 0;
    tb.sort_p1 = c->multi_step_call ? c->sort_deep_p1 : c->sort_p1;
    tb.sort_p2 = c->multi_step_call ? c->sort_deep_p2 : c->sort_p2;
    tb.sort_checked = 1;
    tb.cond_stream = c->cond_stream;
    tb.cond_launches = &c->capture_cond_launches;
}

void ev(nbody_ctx *c, int k) {
    if (c->timing) cudaEventRecord(c->ev[k], c->stream);
}

// One force pass on the resident pos/mass: tree, COM, walk. Asynchronous.
int apply_min_size(nbody_ctx *c, bool want_vmax, unsigned *launches);
int copy_tree_slot(nbody_ctx *c, uint32_t i, bool save);

int force_pass(nbody_ctx *c, int damping, double theta, bool fp64, bool want_vmax, bool track_amax,
               bool want_counts, bool want_pot, const double *pos = nullptr, bool adjoint = false,
               const WalkLaunch *shape = nullptr, bool min_size = false, int save_slot = -1, int restore_slot = -1,
               double *acc64_out = nullptr) {
    uint32_t n = c->n;
    unsigned launches = 1;
    NB_CUDA(launch_reset_pass(c->sc, c->stream));
    tree_inputs(c, n, want_vmax);
    if (pos) c->tb.pos = pos;
    const bool multi = c->nsys > 1 && !c->single_pass && c->sys_total == n;
    c->tb.nsys = multi ? c->nsys : 1;
    c->tb.sys_start = c->sys_start;
    c->tb.sys_id = c->sys_id;
    c->tb.sys_sorted = c->sys_sorted;
    c->tb.sys_root = c->sys_root;
    c->tb.sys_root_node = c->sys_root_node;
    ev(c, 0);
    if (restore_slot >= 0 && !multi) {
        // the octree of these positions was saved by the forward recomputation
        int rc = copy_tree_slot(c, (uint32_t)restore_slot, false);
        if (rc) return rc;
        ev(c, 1);
    } else {
        NB_CUDA(build_octree(c->tb, c->stream, &launches));
        if (min_size && c->p.min_node_size > 0 && n >= 2 && !multi) {
            int rc = apply_min_size(c, want_vmax, &launches);
            if (rc) return rc;
            n = c->n;
        }
        ev(c, 1);
        NB_CUDA(compute_com(c->tb, c->stream, &launches));
        if (save_slot >= 0 && !multi) {
            int rc = copy_tree_slot(c, (uint32_t)save_slot, true);
            if (rc) return rc;
        }
    }
    ev(c, 2);
    WalkArgs a{};
    a.t.n = n;
    a.t.body = c->tb.body;
    a.t.sidx = c->tb.idx_a;
    a.t.onode = c->tb.onode;
    a.t.ochild = c->tb.ochild;
    a.t.ometa = c->tb.ometa;
    a.t.sc = c->sc;
    a.theta = theta;
    a.damping = damping;
    a.single = single(c) ? 1 : 0;
    a.accf = fp64 ? nullptr : (float *)c->acc;
    a.accd = fp64 ? (acc64_out ? acc64_out : (double *)c->acc) : nullptr;
    a.counts = want_counts ? c->counts : nullptr;
    a.pot = want_pot ? c->pot : nullptr;
    a.spill = c->spill;
    a.spill_cap = kSpillCap;
    a.n_groups = multi ? c->ngroups : (n + 31) / 32;
    a.groups = multi ? c->groups : nullptr;
    a.sys_root_node = c->sys_root_node;
    a.sys_root = c->sys_root;
    a.track_max_acc = track_amax ? 1 : 0;
    a.stats = c->walk_stats;
    if (adjoint) {
        a.adjoint = 1;
        a.lamf = (const float *)c->lam;
        a.lamd = c->lam;
        a.gdirf = (float *)c->gdir;
        a.gdird = c->gdir;
        a.adj_node = c->adj_node;
        a.adj_leaf = c->adj_leaf;
        NB_CUDA(cudaMemsetAsync(c->adj_node, 0, 32 * (size_t)n, c->stream));
        NB_CUDA(cudaMemsetAsync(c->adj_leaf, 0, 32 * (size_t)n, c->stream));
    }
    if (n > 0) {
        NB_CUDA(launch_walk(a, fp64, shape ? *shape : fp64 ? c->wl_fp64 : c->wl_mixed, c->stream));
        launches++;
    }
    c->launches += launches;
    ev(c, 3);
    if (!acc64_out) c->have_acc = true;
    return NBODY_OK;
}

// Clears the per-call status bits and the per-call interaction total.
int begin_call(nbody_ctx *c) {
    NB_CUDA(cudaMemsetAsync(&c->sc->status, 0, sizeof(uint32_t), c->stream));
    NB_CUDA(cudaMemsetAsync(&c->sc->interactions_total, 0, sizeof(unsigned long long), c->stream));
    return NBODY_OK;
}

int copy_scalars_back(nbody_ctx *c) {
    NB_CUDA(cudaMemcpyAsync(c->hsc, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    return NBODY_OK;
}

int upload(nbody_ctx *c, uint32_t n, const double *pos, const double *vel, const double *mass) {
    int rc = reserve(c, n);
    if (rc) return rc;
    NB_CUDA(cudaMemcpyAsync(c->pos, pos, 24 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->mass, mass, 8 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if (vel) NB_CUDA(cudaMemcpyAsync(c->vel, vel, 24 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    else NB_CUDA(cudaMemsetAsync(c->vel, 0, 24 * (size_t)n, c->stream));
    c->n = n;
    c->have_state = true;
    c->have_vel = vel != nullptr;
    c->have_acc = false;
    return NBODY_OK;
}

int download_acc(nbody_ctx *c, double *acc) {
    const size_t cnt = 3 * (size_t)c->n;
    if (c->p.precision == NBODY_PRECISION_FP64) {
        NB_CUDA(cudaMemcpyAsync(acc, c->acc, 8 * cnt, cudaMemcpyDeviceToHost, c->stream));
    } else {
        NB_CUDA(launch_acc_to_double((const float *)c->acc, c->acc_out, cnt, c->stream));
        c->launches++;
        NB_CUDA(cudaMemcpyAsync(acc, c->acc_out, 8 * cnt, cudaMemcpyDeviceToHost, c->stream));
    }
    return NBODY_OK;
}

// ---- CUDA graphs ---------------------------------------------------------------
// Everything a captured sequence depends on; a change forces a new capture.
std::vector<unsigned char> graph_key(nbody_ctx *c, uint32_t extra) {
    struct K {
        uint32_t n, nsys, ngroups, extra;
        int sort_p1, sort_p2, walk_stats;
        void *arena, *adj, *sys, *stream;
        nbody_params p;
        WalkLaunch wm, wf;
    } k;
    std::memset(&k, 0, sizeof k);
    k.n = c->n; k.nsys = c->nsys; k.ngroups = c->ngroups; k.extra = extra;
    k.sort_p1 = c->multi_step_call ? c->sort_deep_p1 : c->sort_p1;
    k.sort_p2 = c->multi_step_call ? c->sort_deep_p2 : c->sort_p2; k.walk_stats = c->walk_stats;
    k.arena = c->arena; k.adj = c->adj_arena; k.sys = c->sys_arena; k.stream = (void *)c->stream;
    k.p = c->p; k.wm = c->wl_mixed; k.wf = c->wl_fp64;
    const unsigned char *b = (const unsigned char *)&k;
    return std::vector<unsigned char>(b, b + sizeof k);
}

void drop_graph(cudaGraphExec_t &g) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
}

void drop_graphs(nbody_ctx *c) {
    drop_graph(c->step_exec);
    for (auto &g : c->rec_exec) drop_graph(g);
    for (auto &g : c->adj_exec) drop_graph(g);
    c->rec_exec.clear(); c->adj_exec.clear();
    c->rec_launches.clear(); c->adj_launches.clear();
    c->step_key.clear(); c->adj_key.clear();
}

// Captures what `body` enqueues on the context stream into an executable graph.
// Returns false (nothing captured, no error left behind) when capture is not
// possible on this stream; the caller then launches directly.
template <class F>
bool capture(nbody_ctx *c, cudaGraphExec_t *out, unsigned *launches, F &&body) {
    *out = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const unsigned long long l0 = c->launches;
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    bool ok = rc == NBODY_OK && e == cudaSuccess && g;
    if (ok) ok = cudaGraphInstantiate(out, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    *launches = (unsigned)(c->launches - l0);
    c->launches = l0;
    if (!ok) {
        cudaGetLastError();
        *out = nullptr;
    }
    return ok;
}

// ---- merging ------------------------------------------------------------------
bool merging(const nbody_ctx *c) { return c->p.collide || c->p.min_node_size > 0; }

int reserve_merge(nbody_ctx *c) {
    if (c->merge_arena && c->merge_cap >= c->cap) return NBODY_OK;
    const size_t N = c->cap;
    MergeBufs &m = c->mb;
    struct Piece { void **dst; size_t bytes; };
    Piece pieces[] = {
        {(void **)&m.label, 4 * N}, {(void **)&m.rep, 4 * N}, {(void **)&m.flag, 4 * N}, {(void **)&m.offs, 4 * N},
        {(void **)&m.scan_tmp, 4 * ((N + 4095) / 4096 + 8)},
        {(void **)&m.mpos, 24 * N}, {(void **)&m.mvel, 24 * N}, {(void **)&m.mmass, 8 * N},
        {(void **)&m.pos2, 24 * N}, {(void **)&m.vel2, 24 * N}, {(void **)&m.mass2, 8 * N}, {(void **)&m.acc2, 24 * N},
        {(void **)&m.skey_a, 8 * N}, {(void **)&m.skey_b, 8 * N}, {(void **)&m.sidx_a, 4 * N},
        {(void **)&m.sidx_b, 4 * N}, {(void **)&m.sort_scratch, sort_scratch_bytes(c->cap)},
        {(void **)&m.counters, 4 * kMcCount},
    };
    size_t total = 0;
    for (auto &pc : pieces) total += align256(pc.bytes);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    if (c->merge_arena) NB_CUDA(cudaFree(c->merge_arena));
    c->merge_arena = nullptr;
    c->merge_cap = 0;
    cudaError_t e = cudaMalloc(&c->merge_arena, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->merge_arena = nullptr;
        return fail(NBODY_ERR_OOM, "merge buffers (%s)", cudaGetErrorString(e));
    }
    char *p = (char *)c->merge_arena;
    for (auto &pc : pieces) {
        *pc.dst = p;
        p += align256(pc.bytes);
    }
    c->merge_bytes = total;
    c->merge_cap = c->cap;
    if (!c->hcounters) {
        if (cudaMallocHost(&c->hcounters, 4 * kMcCount) != cudaSuccess) {
            cudaGetLastError();
            c->hcounters = nullptr;
            return fail(NBODY_ERR_OOM, "pinned counters%s");
        }
    }
    return NBODY_OK;
}

int reserve_pairs(nbody_ctx *c, uint32_t need) {
    if (c->pairs && c->mb.pair_cap >= need) return NBODY_OK;
    uint32_t cap = std::max<uint32_t>(need + need / 2, 4096u);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    if (c->pairs) NB_CUDA(cudaFree(c->pairs));
    c->pairs = nullptr;
    c->mb.pair_cap = 0;
    cudaError_t e = cudaMalloc(&c->pairs, sizeof(uint2) * (size_t)cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->pairs = nullptr;
        return fail(NBODY_ERR_OOM, "collision pair buffer (%s)", cudaGetErrorString(e));
    }
    c->mb.pairs = c->pairs;
    c->mb.pair_cap = cap;
    return NBODY_OK;
}

// Waits for the stream and reads the merge counters; fails on a merge status bit.
int read_counters(nbody_ctx *c) {
    NB_CUDA(cudaMemcpyAsync(c->hcounters, c->mb.counters, 4 * kMcCount, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    if (c->hcounters[kMcStatus])
        return fail(NBODY_ERR_CUDA, "particle merging failed (status bits %s)",
                    c->hcounters[kMcStatus] & kMergeStatusSort ? "sort" : "tree/union");
    return NBODY_OK;
}

Tree tree_view(nbody_ctx *c) {
    Tree t{};
    t.n = c->n;
    t.body = c->tb.body;
    t.sidx = c->tb.idx_a;
    t.onode = c->tb.onode;
    t.ochild = c->tb.ochild;
    t.ometa = c->tb.ometa;
    t.sc = c->sc;
    return t;
}

// Compacts to the kept particles (merged values at the representatives) and
// adopts the new count; returns the number removed.
int adopt_compaction(nbody_ctx *c, bool fp64, unsigned *launches, uint64_t *removed) {
    const uint32_t n = c->n;
    NB_CUDA(merge_compact(c->mb, n, c->pos, c->vel, c->mass, c->acc, fp64, c->stream, launches));
    int rc = read_counters(c);
    if (rc) return rc;
    const uint32_t kept = c->hcounters[kMcKept];
    if (kept == 0 || kept > n) return fail(NBODY_ERR_CUDA, "particle merging kept an impossible count%s");
    NB_CUDA(cudaMemcpyAsync(c->pos, c->mb.pos2, 24 * (size_t)kept, cudaMemcpyDeviceToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->vel, c->mb.vel2, 24 * (size_t)kept, cudaMemcpyDeviceToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->mass, c->mb.mass2, 8 * (size_t)kept, cudaMemcpyDeviceToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->acc, c->mb.acc2, (fp64 ? 24 : 12) * (size_t)kept, cudaMemcpyDeviceToDevice,
                            c->stream));
    *removed = n - kept;
    c->n = kept;
    c->have_fwd = false;
    return NBODY_OK;
}

// apply_minimum_size on the octree just built; rebuilds it in the same root
// cube when anything merged (the reference keeps its root).
int apply_min_size(nbody_ctx *c, bool want_vmax, unsigned *launches) {
    int rc = reserve_merge(c);
    if (rc) return rc;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    NB_CUDA(merge_begin(c->mb, c->n, c->stream, launches));
    NB_CUDA(merge_min_size(c->mb, tree_view(c), c->tb.oparent, c->vel, c->p.min_node_size, c->stream, launches));
    if ((rc = read_counters(c))) return rc;
    if (c->hcounters[kMcGroups] == 0) return NBODY_OK;
    uint64_t removed = 0;
    if ((rc = adopt_compaction(c, fp64, launches, &removed))) return rc;
    c->merged_min_size += removed;
    tree_inputs(c, c->n, want_vmax);
    c->tb.keep_root = 1;
    cudaError_t e = build_octree(c->tb, c->stream, launches);
    c->tb.keep_root = 0;
    NB_CUDA(e);
    return NBODY_OK;
}

// Collision capture on the octree of the force pass just run, then the merge.
int apply_collisions(nbody_ctx *c, unsigned *launches) {
    if (c->n < 2) return NBODY_OK;
    int rc = reserve_merge(c);
    if (rc) return rc;
    if ((rc = reserve_pairs(c, 4096))) return rc;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    uint32_t np = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        NB_CUDA(merge_begin(c->mb, c->n, c->stream, launches));
        NB_CUDA(collide_find(c->mb, tree_view(c), c->tb.oparent, c->p.theta, c->p.collision_range, c->stream,
                             launches));
        if ((rc = read_counters(c))) return rc;
        np = c->hcounters[kMcPairs];
        if (np <= c->mb.pair_cap) break;
        if ((rc = reserve_pairs(c, np))) return rc;  // found more than fit: grow and search again
    }
    c->collision_pairs += np;
    if (np == 0) return NBODY_OK;
    if (np > c->mb.pair_cap) return fail(NBODY_ERR_CAPACITY, "collision pairs exceed the buffer%s");
    NB_CUDA(collide_components(c->mb, c->n, np, c->stream, launches));
    if ((rc = read_counters(c))) return rc;
    NB_CUDA(collide_fold(c->mb, c->hcounters[kMcInvolved], c->pos, c->vel, c->mass, c->stream, launches));
    uint64_t removed = 0;
    if ((rc = adopt_compaction(c, fp64, launches, &removed))) return rc;
    c->merged_collisions += removed;
    if (c->p.adaptive) {
        NB_CUDA(launch_maxima(c->acc, fp64, c->vel, c->n, c->sc, c->stream));
        *launches += 1;
    }
    return NBODY_OK;
}

int one_step(nbody_ctx *c) {
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    StepParams sp{c->p.dt, c->p.adaptive, c->p.min_adaptive_dt, c->p.max_pos_change, c->p.max_vel_change,
                  single(c)};
    const bool merge = merging(c);
    int rc = force_pass(c, c->p.damping, c->p.theta, fp64, c->p.adaptive != 0, c->p.adaptive != 0, false, false,
                        nullptr, false, nullptr, merge);
    if (rc) return rc;
    if (merge && c->p.collide) {
        unsigned launches = 0;
        rc = apply_collisions(c, &launches);
        c->launches += launches;
        if (rc) return rc;
    }
    NB_CUDA(launch_update(c->pos, c->vel, c->acc, fp64, c->n, sp, c->sc, c->stream));
    c->launches++;
    return NBODY_OK;
}

int run_steps(nbody_ctx *c, uint32_t nsteps) {
    if (c->use_graphs && !c->timing && !merging(c)) {  // merging changes n: launched step by step
        auto key = graph_key(c, 0);
        if (!c->step_exec || key != c->step_key) {
            drop_graph(c->step_exec);
            c->step_key.clear();
            c->capture_cond_launches = 0;
            if (capture(c, &c->step_exec, &c->step_launches, [&] { return one_step(c); })) c->step_key = key;
            c->step_cond_launches = c->capture_cond_launches;
        }
        if (c->step_exec) {
            // the conditional node's kernels are counted when a replay ran them (check_status)
            for (uint32_t s = 0; s < nsteps; s++) {
                NB_CUDA(cudaGraphLaunch(c->step_exec, c->stream));
                c->launches += c->step_launches - c->step_cond_launches;
            }
            c->replayed_cond_launches = c->step_cond_launches;
            return NBODY_OK;
        }
    }
    for (uint32_t s = 0; s < nsteps; s++) {
        int rc = one_step(c);
        if (rc) return rc;
        ev(c, 4);
    }
    return NBODY_OK;
}

// Adjoint buffers for n particles, `seg` positions per checkpoint segment and
// `nckpt` checkpoints of (pos, vel).
// Bytes of one saved octree of n particles (tree_slot_ptrs below).
size_t tree_slot_bytes(uint32_t n) {
    const size_t N = n;
    return align256(32 * N) + align256(4 * N) + align256(32 * N) + align256(32 * N) + align256(4 * N) +
           align256(4 * N) + align256(4 * N) + align256(32);
}

struct TreeSlot {
    double4 *body, *onode;
    uint32_t *sidx;
    int32_t *ochild, *ometa, *oparent, *leaf_oparent;
    double *root;  // root_center[3], root_side
};

TreeSlot tree_slot_ptrs(nbody_ctx *c, uint32_t i) {
    const size_t N = c->n;
    char *p = (char *)c->tree_slots + tree_slot_bytes(c->n) * i;
    TreeSlot t;
    t.body = (double4 *)p; p += align256(32 * N);
    t.sidx = (uint32_t *)p; p += align256(4 * N);
    t.onode = (double4 *)p; p += align256(32 * N);
    t.ochild = (int32_t *)p; p += align256(32 * N);
    t.ometa = (int32_t *)p; p += align256(4 * N);
    t.oparent = (int32_t *)p; p += align256(4 * N);
    t.leaf_oparent = (int32_t *)p; p += align256(4 * N);
    t.root = (double *)p;
    return t;
}

// Copies the octree just built to slot i (save) or slot i to the build buffers.
int copy_tree_slot(nbody_ctx *c, uint32_t i, bool save) {
    const size_t N = c->n, M = N > 0 ? N - 1 : 0;
    const TreeSlot t = tree_slot_ptrs(c, i);
    TreeBuild &tb = c->tb;
    struct Pair { void *slot; void *live; size_t bytes; } pairs[] = {
        {t.body, tb.body, 32 * N}, {t.sidx, tb.idx_a, 4 * N}, {t.onode, tb.onode, 32 * M},
        {t.ochild, tb.ochild, 32 * M}, {t.ometa, tb.ometa, 4 * M}, {t.oparent, tb.oparent, 4 * M},
        {t.leaf_oparent, tb.leaf_oparent, 4 * N}, {t.root, c->sc->root_center, 32},
    };
    for (auto &q : pairs) {
        if (!q.bytes) continue;
        NB_CUDA(cudaMemcpyAsync(save ? q.slot : q.live, save ? q.live : q.slot, q.bytes, cudaMemcpyDeviceToDevice,
                                c->stream));
    }
    return NBODY_OK;
}

// Adjoint buffers for n particles, `seg` positions per checkpoint segment and
// `nckpt` checkpoints of (pos, vel); with `slots`, room for `seg` saved octrees
// as well when the device has it.
int reserve_adjoint(nbody_ctx *c, uint32_t n, uint32_t seg, uint32_t nckpt, bool slots = false) {
    const size_t N = n;
    struct Piece { double **dst; size_t bytes; };
    Piece pieces[] = {
        {&c->lx, 24 * N}, {&c->lv, 24 * N}, {&c->lm, 8 * N}, {&c->lam, 24 * N}, {&c->gdir, 24 * N},
        {&c->adj_node, 32 * N}, {&c->adj_leaf, 32 * N}, {&c->vel_work, 24 * N},
        {&c->seg_pos, 24 * N * seg}, {&c->ckpt, 48 * N * nckpt},
    };
    size_t total = 0;
    for (auto &pc : pieces) total += align256(pc.bytes);
    size_t with_slots = total;
    if (slots && c->nsys <= 1) {
        size_t free_b = 0, tot_b = 0;
        if (cudaMemGetInfo(&free_b, &tot_b) != cudaSuccess) cudaGetLastError();
        const size_t extra = tree_slot_bytes(n) * seg;
        // keep a margin: the slots are an optimisation, never worth an allocation failure
        if (extra + total < c->adj_bytes || extra + total < free_b / 2) with_slots = total + extra;
    }
    if (with_slots > c->adj_bytes) {
        NB_CUDA(cudaStreamSynchronize(c->stream));
        if (c->adj_arena) NB_CUDA(cudaFree(c->adj_arena));
        c->adj_arena = nullptr;
        c->adj_bytes = 0;
        cudaError_t e = cudaMalloc(&c->adj_arena, with_slots);
        if (e != cudaSuccess && with_slots > total) {
            cudaGetLastError();
            with_slots = total;
            e = cudaMalloc(&c->adj_arena, total);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->adj_arena = nullptr;
            return fail(NBODY_ERR_OOM, "adjoint buffers (%s)", cudaGetErrorString(e));
        }
        c->adj_bytes = with_slots;
    }
    char *p = (char *)c->adj_arena;
    for (auto &pc : pieces) {
        *pc.dst = (double *)p;
        p += align256(pc.bytes);
    }
    c->tree_slots = nullptr;
    c->n_slots = 0;
    if (with_slots > total) {
        c->tree_slots = (double *)p;
        c->n_slots = seg;
    }
    return NBODY_OK;
}

// One reverse force step at positions `pos` with cotangent c->lam (dL/da):
// tree and COM at pos, the adjoint walk over the same decisions, then the node
// cotangents distributed to particles; adds into c->lx and c->lm.
int adjoint_force(nbody_ctx *c, const double *pos, int damping, double theta, bool fp64, int restore_slot = -1) {
    int rc = force_pass(c, damping, theta, fp64, false, false, false, false, pos, true, nullptr, false, -1, restore_slot);
    if (rc) return rc;
    NB_CUDA(launch_adj_distribute(c->tb.body, c->tb.idx_a, c->tb.leaf_oparent, c->tb.oparent, c->tb.onode,
                                  c->adj_node, c->adj_leaf, c->gdir, fp64, fp64 ? nullptr : &c->sc->lam_scale, c->lx,
                                  c->lm, c->n, c->stream));
    c->launches++;
    return NBODY_OK;
}

// ---- autotuner ----------------------------------------------------------------
// Times the walk on the resident state for every block shape (1, 2 or 4 warps
// per block; all or all-but-one resident blocks per SM) and keeps the fastest
// for this context's precision. Tree and COM are rebuilt per candidate so each
// walk starts from the same state; only the walk is timed (CUDA events, best of 3).
std::vector<unsigned char> tune_key(nbody_ctx *c) {
    struct K { uint32_t n_bucket, nsys; int precision, damping; double theta; } k;
    std::memset(&k, 0, sizeof k);
    uint32_t b = 1;
    while (b < c->n) b <<= 1;
    k.n_bucket = b; k.nsys = c->nsys; k.precision = c->p.precision; k.damping = c->p.damping; k.theta = c->p.theta;
    const unsigned char *p = (const unsigned char *)&k;
    return std::vector<unsigned char>(p, p + sizeof k);
}

int autotune(nbody_ctx *c) {
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    const int saved_timing = c->timing;
    c->timing = 1;
    WalkLaunch best = fp64 ? c->wl_fp64 : c->wl_mixed;
    float best_ms = 1e30f;
    int rc = NBODY_OK;
    for (unsigned w : {1u, 2u, 4u}) {
        int maxb = 0;
        if (walk_max_blocks_per_sm(fp64, w, &maxb) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        for (int bps = maxb; bps >= 1 && bps >= maxb - 1; bps--) {
            WalkLaunch shape{};
            if (walk_launch_shape(fp64, c->p.device, w, (unsigned)bps, &shape) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if ((size_t)shape.blocks * shape.warps > c->max_walk_warps) continue;
            float ms = 1e30f;
            for (int r = 0; r < 3 && rc == NBODY_OK; r++) {
                rc = force_pass(c, c->p.damping, c->p.theta, fp64, false, false, false, false, nullptr, false, &shape);
                if (rc) break;
                if ((rc = copy_scalars_back(c))) break;
                if ((rc = check_status(c))) break;
                ms = std::min(ms, c->stats.ms_walk);
            }
            if (rc) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = shape;
            }
        }
        if (rc) break;
    }
    c->timing = saved_timing;
    if (rc) return rc;
    if (fp64) c->wl_fp64 = best;
    else c->wl_mixed = best;
    drop_graphs(c);
    c->tuned_key = tune_key(c);
    return NBODY_OK;
}

int maybe_autotune(nbody_ctx *c) {
    if (!c->p.autotune || c->n < 2) return NBODY_OK;
    if (tune_key(c) == c->tuned_key) return NBODY_OK;
    return autotune(c);
}

// Runs `body` through the graph cached at slot i (capturing it on first use).
template <class F>
int run_cached(nbody_ctx *c, std::vector<cudaGraphExec_t> &execs, std::vector<unsigned> &launches, uint32_t i,
               F &&body) {
    if (c->use_graphs && !c->timing) {
        if (execs.size() <= i) {
            execs.resize(i + 1, nullptr);
            launches.resize(i + 1, 0);
        }
        if (!execs[i]) capture(c, &execs[i], &launches[i], body);
        if (execs[i]) {
            NB_CUDA(cudaGraphLaunch(execs[i], c->stream));
            c->launches += launches[i];
            return NBODY_OK;
        }
    }
    return body();
}

#define CTX_OR_FAIL(c)                                                 \
    do {                                                               \
        if (!(c)) return fail(NBODY_ERR_INVALID, "context is null%s"); \
        int rc_ = set_device(c);                                       \
        if (rc_) return rc_;                                           \
    } while (0)

}  // namespace

extern "C" {

void nbody_default_params(nbody_params *p) {
    if (!p) return;
    p->theta = 0.5;       // src/main.cpp:1327
    p->dt = 0.0333;       // src/main.cpp:1328
    p->damping = 0;       // src/main.cpp:1343
    p->adaptive = 0;      // README.md:54
    p->min_adaptive_dt = 0.00333;  // README.md:56
    p->max_pos_change = 3;         // README.md:58
    p->max_vel_change = 3;         // README.md:60
    p->precision = NBODY_PRECISION_MIXED;
    p->device = 0;
    p->autotune = 0;
    p->collide = 0;              // src/main.cpp:1353
    p->collision_range = 0.01;   // src/main.cpp:1354
    p->min_node_size = 0.0;      // src/main.cpp:1355
    p->datatype_bytes = 8;       // the DOUBLE build (src/vector.h:4-13)
}

int nbody_create(const nbody_params *p, nbody_ctx **out) {
    if (!out) return fail(NBODY_ERR_INVALID, "out is null%s");
    *out = nullptr;
    int rc = check_params(p);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p->device || p->device < 0) {
        cudaGetLastError();
        return fail(NBODY_ERR_NO_DEVICE, "no CUDA device with ordinal %s", "requested");
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, p->device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return fail(NBODY_ERR_NO_DEVICE, "device is not sm_100 (this library is built for sm_100a only)%s");
    }
    nbody_ctx *c = new (std::nothrow) nbody_ctx();
    if (!c) return fail(NBODY_ERR_OOM, "host allocation failed%s");
    c->p = *p;
    auto cleanup = [&](int code) { nbody_destroy(c); return code; };
    if ((rc = set_device(c))) return cleanup(rc);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(NBODY_ERR_CUDA, "stream creation failed%s"));
    c->own_stream = true;
    if (cudaStreamCreateWithFlags(&c->cond_stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(NBODY_ERR_CUDA, "stream creation failed%s"));
    if (cudaMalloc(&c->sc, sizeof(DevScalars)) != cudaSuccess) return cleanup(fail(NBODY_ERR_OOM, "scalars%s"));
    if (cudaMemset(c->sc, 0, sizeof(DevScalars)) != cudaSuccess) return cleanup(fail(NBODY_ERR_CUDA, "memset%s"));
    if (cudaMallocHost(&c->hsc, sizeof(DevScalars)) != cudaSuccess) return cleanup(fail(NBODY_ERR_OOM, "pinned%s"));
    std::memset(c->hsc, 0, sizeof(DevScalars));
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return cleanup(fail(NBODY_ERR_CUDA, "event%s"));
    if (walk_launch_shape(false, p->device, kWalkWarps, 0, &c->wl_mixed) != cudaSuccess ||
        walk_launch_shape(true, p->device, kWalkWarps, 0, &c->wl_fp64) != cudaSuccess)
        return cleanup(fail(NBODY_ERR_CUDA, "walk kernel configuration failed (%s)",
                            cudaGetErrorString(cudaGetLastError())));
    // spill regions for the largest resident warp count any tuned shape can have
    for (unsigned w : {1u, 2u, 4u})
        for (int fp = 0; fp < 2; fp++) {
            int mb = 0;
            if (walk_max_blocks_per_sm(fp != 0, w, &mb) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            c->max_walk_warps = std::max(c->max_walk_warps, (unsigned)(prop.multiProcessorCount * mb * (int)w));
        }
    *out = c;
    return NBODY_OK;
}

int nbody_destroy(nbody_ctx *c) {
    if (!c) return NBODY_OK;
    cudaSetDevice(c->p.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    if (c->arena) cudaFree(c->arena);
    if (c->adj_arena) cudaFree(c->adj_arena);
    if (c->sys_arena) cudaFree(c->sys_arena);
    if (c->img_arena) cudaFree(c->img_arena);
    if (c->merge_arena) cudaFree(c->merge_arena);
    if (c->direct_arena) cudaFree(c->direct_arena);
    if (c->pairs) cudaFree(c->pairs);
    if (c->hcounters) cudaFreeHost(c->hcounters);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->cond_stream) cudaStreamDestroy(c->cond_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_mass) cudaEventDestroy(c->ev_mass);
    if (c->ev_vel) cudaEventDestroy(c->ev_vel);
    if (c->sc) cudaFree(c->sc);
    if (c->hsc) cudaFreeHost(c->hsc);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return NBODY_OK;
}

int nbody_set_params(nbody_ctx *c, const nbody_params *p) {
    CTX_OR_FAIL(c);
    int rc = check_params(p);
    if (rc) return rc;
    if (p->device != c->p.device) return fail(NBODY_ERR_INVALID, "device cannot change on a live context%s");
    if (p->precision != c->p.precision) c->have_acc = false;
    c->p = *p;
    return NBODY_OK;
}

int nbody_set_stream(nbody_ctx *c, void *stream) {
    CTX_OR_FAIL(c);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return NBODY_OK;
}

int nbody_autotune(nbody_ctx *c) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (c->n < 2) return NBODY_OK;
    int rc = begin_call(c);
    if (rc) return rc;
    return autotune(c);
}

int nbody_set_graphs(nbody_ctx *c, int enabled) {
    CTX_OR_FAIL(c);
    NB_CUDA(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->use_graphs = enabled != 0;
    return NBODY_OK;
}

int nbody_set_timing(nbody_ctx *c, int enabled) {
    CTX_OR_FAIL(c);
    c->timing = enabled ? 1 : 0;
    return NBODY_OK;
}

int nbody_set_walk_stats(nbody_ctx *c, int enabled) {
    CTX_OR_FAIL(c);
    c->walk_stats = enabled ? 1 : 0;
    return NBODY_OK;
}

int nbody_barnes_hut(nbody_ctx *c, uint32_t n, const double *pos, const double *mass, int damping, double theta,
                     double *acc_out, uint32_t *counts_out) {
    CTX_OR_FAIL(c);
    if (n > kMaxParticles) return fail(NBODY_ERR_INVALID, "n exceeds the 2^28 particle limit%s");
    if (n && (!pos || !mass || !acc_out)) return fail(NBODY_ERR_INVALID, "null array%s");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(NBODY_ERR_INVALID, "theta must be finite and > 0%s");
    if (n == 0) return NBODY_OK;
    int rc = upload(c, n, pos, nullptr, mass);
    if (rc) return rc;
    if ((rc = begin_call(c))) return rc;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    c->single_pass = true;
    rc = force_pass(c, damping ? 1 : 0, theta, fp64, false, false, counts_out != nullptr, false);
    c->single_pass = false;
    if (rc) return rc;
    ev(c, 4);
    if ((rc = download_acc(c, acc_out))) return rc;
    if (counts_out) NB_CUDA(cudaMemcpyAsync(counts_out, c->counts, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_set_systems(nbody_ctx *c, uint32_t nsys, const uint32_t *counts) {
    CTX_OR_FAIL(c);
    if (nsys == 0 || nsys > 65536 || (nsys > 1 && !counts)) return fail(NBODY_ERR_INVALID, "1 <= nsys <= 65536%s");
    if (nsys == 1) {
        c->nsys = 1;
        c->sys_total = 0;
        return NBODY_OK;
    }
    uint64_t total = 0;
    uint32_t ngroups = 0;
    for (uint32_t k = 0; k < nsys; k++) {
        if (counts[k] == 0) return fail(NBODY_ERR_INVALID, "every system needs at least one particle%s");
        total += counts[k];
        ngroups += (counts[k] + 31) / 32;
    }
    if (total > kMaxParticles) return fail(NBODY_ERR_INVALID, "total exceeds the 2^28 particle limit%s");
    const size_t N = total;
    struct Piece { void **dst; size_t bytes; };
    Piece pieces[] = {{(void **)&c->sys_start, 4 * ((size_t)nsys + 1)}, {(void **)&c->sys_id, 4 * N},
                      {(void **)&c->sys_sorted, 4 * N}, {(void **)&c->groups, 16 * (size_t)ngroups},
                      {(void **)&c->sys_root, 32 * (size_t)nsys}, {(void **)&c->sys_root_node, 4 * (size_t)nsys}};
    size_t bytes = 0;
    for (auto &pc : pieces) bytes += align256(pc.bytes);
    if (bytes > c->sys_bytes) {
        NB_CUDA(cudaStreamSynchronize(c->stream));
        if (c->sys_arena) NB_CUDA(cudaFree(c->sys_arena));
        c->sys_arena = nullptr;
        c->sys_bytes = 0;
        cudaError_t e = cudaMalloc(&c->sys_arena, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(NBODY_ERR_OOM, "system tables (%s)", cudaGetErrorString(e));
        }
        c->sys_bytes = bytes;
    }
    char *p = (char *)c->sys_arena;
    for (auto &pc : pieces) {
        *pc.dst = p;
        p += align256(pc.bytes);
    }
    std::vector<uint32_t> start(nsys + 1), sid(N);
    std::vector<int4> groups;
    groups.reserve(ngroups);
    start[0] = 0;
    for (uint32_t k = 0; k < nsys; k++) {
        start[k + 1] = start[k] + counts[k];
        for (uint32_t i = start[k]; i < start[k + 1]; i++) sid[i] = k;
        for (uint32_t o = 0; o < counts[k]; o += 32)
            groups.push_back(make_int4((int)(start[k] + o), (int)std::min(32u, counts[k] - o), (int)k, 0));
    }
    NB_CUDA(cudaMemcpyAsync(c->sys_start, start.data(), 4 * start.size(), cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->sys_id, sid.data(), 4 * N, cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(cudaMemcpyAsync(c->groups, groups.data(), 16 * groups.size(), cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    c->nsys = nsys;
    c->sys_total = (uint32_t)total;
    c->ngroups = ngroups;
    return NBODY_OK;
}

int nbody_set_particles(nbody_ctx *c, uint32_t n, const double *pos, const double *vel, const double *mass) {
    CTX_OR_FAIL(c);
    if (n > kMaxParticles) return fail(NBODY_ERR_INVALID, "n exceeds the 2^28 particle limit%s");
    if (c->nsys > 1 && n != c->sys_total)
        return fail(NBODY_ERR_INVALID, "n differs from the total of the systems declared by nbody_set_systems%s");
    if (n && (!pos || !mass)) return fail(NBODY_ERR_INVALID, "null array%s");
    int rc = upload(c, n, pos, vel, mass);
    if (rc) return rc;
    NB_CUDA(cudaStreamSynchronize(c->stream));
    c->have_vel = true;  // a null vel means zero velocities
    return NBODY_OK;
}

int nbody_get_particles(nbody_ctx *c, double *pos, double *vel, double *acc) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (pos) NB_CUDA(cudaMemcpyAsync(pos, c->pos, 24 * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    if (vel) NB_CUDA(cudaMemcpyAsync(vel, c->vel, 24 * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    if (acc) {
        if (!c->have_acc) return fail(NBODY_ERR_STATE, "no forces computed yet%s");
        int rc = download_acc(c, acc);
        if (rc) return rc;
    }
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NBODY_OK;
}

int nbody_get_masses(nbody_ctx *c, double *mass) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (!mass) return fail(NBODY_ERR_INVALID, "mass is null%s");
    NB_CUDA(cudaMemcpyAsync(mass, c->mass, 8 * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NBODY_OK;
}

int nbody_compute_forces(nbody_ctx *c) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (c->n == 0) return NBODY_OK;
    int rc = begin_call(c);
    if (rc) return rc;
    rc = force_pass(c, c->p.damping, c->p.theta, c->p.precision == NBODY_PRECISION_FP64, false, false, false, false);
    if (rc) return rc;
    ev(c, 4);
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_step(nbody_ctx *c, uint32_t nsteps) {
    CTX_OR_FAIL(c);
    if (!c->have_state || !c->have_vel) return fail(NBODY_ERR_STATE, "particles with velocities must be set first%s");
    if (merging(c) && c->nsys > 1)
        return fail(NBODY_ERR_INVALID, "collisions and min_node_size need a single system%s");
    c->merged_min_size = c->merged_collisions = c->collision_pairs = 0;
    if (c->n == 0 || nsteps == 0) return NBODY_OK;
    MultiStepCall scope(c, nsteps > 1);
    int rc = begin_call(c);
    if (rc) return rc;
    if ((rc = maybe_autotune(c))) return rc;
    rc = run_steps(c, nsteps);
    if (rc) return rc;
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_step_host(nbody_ctx *c, uint32_t n, double *pos, double *vel, const double *mass, uint32_t nsteps) {
    CTX_OR_FAIL(c);
    if (n > kMaxParticles) return fail(NBODY_ERR_INVALID, "n exceeds the 2^28 particle limit%s");
    if (n && (!pos || !vel || !mass)) return fail(NBODY_ERR_INVALID, "null array%s");
    if (merging(c))
        return fail(NBODY_ERR_INVALID, "merging changes n: use nbody_set_particles, nbody_step, nbody_get_particles%s");
    if (n == 0) return NBODY_OK;
    MultiStepCall scope(c, nsteps > 1);
    int rc;
    if (n >= kOverlapMin && nsteps > 0) {
        // Positions first: the root cube, keys and sort need nothing else. The
        // masses (first read when the sorted bodies are gathered) and then the
        // velocities (first read by the update) cross on a second stream while
        // the first force pass runs.
        if ((rc = reserve(c, n))) return rc;
        if (!c->aux_stream) {
            NB_CUDA(cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking));
            NB_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
            NB_CUDA(cudaEventCreateWithFlags(&c->ev_mass, cudaEventDisableTiming));
            NB_CUDA(cudaEventCreateWithFlags(&c->ev_vel, cudaEventDisableTiming));
        }
        // The second stream's copies start once the positions are in, so that they
        // do not share the host link with them.
        NB_CUDA(cudaMemcpyAsync(c->pos, pos, 24 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
        NB_CUDA(cudaEventRecord(c->ev_fork, c->stream));
        NB_CUDA(cudaStreamWaitEvent(c->aux_stream, c->ev_fork, 0));
        NB_CUDA(cudaMemcpyAsync(c->mass, mass, 8 * (size_t)n, cudaMemcpyHostToDevice, c->aux_stream));
        NB_CUDA(cudaEventRecord(c->ev_mass, c->aux_stream));
        NB_CUDA(cudaMemcpyAsync(c->vel, vel, 24 * (size_t)n, cudaMemcpyHostToDevice, c->aux_stream));
        NB_CUDA(cudaEventRecord(c->ev_vel, c->aux_stream));
        c->n = n;
        c->have_state = c->have_vel = true;
        c->have_acc = false;
        if ((rc = begin_call(c))) {
            NB_CUDA(cudaStreamWaitEvent(c->stream, c->ev_vel, 0));
            return rc;
        }
        const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
        StepParams sp{c->p.dt, c->p.adaptive, c->p.min_adaptive_dt, c->p.max_pos_change, c->p.max_vel_change,
                      single(c)};
        c->mass_pending = c->ev_mass;
        rc = force_pass(c, c->p.damping, c->p.theta, fp64, false, false, false, false);
        c->mass_pending = nullptr;
        if (rc) {
            NB_CUDA(cudaStreamWaitEvent(c->stream, c->ev_vel, 0));
            return rc;
        }
        NB_CUDA(cudaStreamWaitEvent(c->stream, c->ev_vel, 0));
        if (c->p.adaptive) {
            NB_CUDA(launch_maxima(c->acc, fp64, c->vel, n, c->sc, c->stream));
            c->launches++;
        }
        NB_CUDA(launch_update(c->pos, c->vel, c->acc, fp64, n, sp, c->sc, c->stream));
        c->launches++;
        if (nsteps > 1 && (rc = run_steps(c, nsteps - 1))) return rc;
    } else {
        if ((rc = upload(c, n, pos, vel, mass))) return rc;
        c->have_vel = true;
        if ((rc = begin_call(c))) return rc;
        if ((rc = run_steps(c, nsteps))) return rc;
    }
    NB_CUDA(cudaMemcpyAsync(pos, c->pos, 24 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaMemcpyAsync(vel, c->vel, 24 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_device_view_get(nbody_ctx *c, nbody_device_view *out) {
    CTX_OR_FAIL(c);
    if (!out) return fail(NBODY_ERR_INVALID, "out is null%s");
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    out->n = c->n;
    out->pos = c->pos;
    out->vel = c->vel;
    out->mass = c->mass;
    out->acc = c->acc;
    out->acc_is_double = c->p.precision == NBODY_PRECISION_FP64;
    return NBODY_OK;
}

int nbody_get_stats(nbody_ctx *c, nbody_stats *out) {
    if (!c || !out) return fail(NBODY_ERR_INVALID, "null argument%s");
    *out = c->stats;
    return NBODY_OK;
}

int nbody_get_diagnostics(nbody_ctx *c, nbody_diagnostics *out) {
    CTX_OR_FAIL(c);
    if (!out) return fail(NBODY_ERR_INVALID, "out is null%s");
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    std::memset(out, 0, sizeof *out);
    if (c->n == 0) return NBODY_OK;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    int rc = begin_call(c);
    if (rc) return rc;
    // The potentials come from the FP64 form of the walk in both precisions: the
    // same opening decisions, FP64 pair terms and sums. A MIXED context keeps its
    // accelerations; the pass writes its FP64 ones to scratch.
    rc = force_pass(c, c->p.damping, c->p.theta, true, false, false, false, true, nullptr, false, nullptr, false, -1,
                    -1, fp64 ? nullptr : c->acc_out);
    if (rc) return rc;
    ev(c, 4);
    NB_CUDA(launch_diag(c->pos, c->vel, c->mass, c->pot, c->n, c->diag_partial, kDiagBlocks, c->sc, c->stream));
    c->launches++;
    if ((rc = copy_scalars_back(c))) return rc;
    if ((rc = check_status(c))) return rc;
    const double *d = c->hsc->diag;
    out->kinetic = d[0];
    out->potential = d[1];
    for (int k = 0; k < 3; k++) {
        out->momentum[k] = d[2 + k];
        out->angular_momentum[k] = d[5 + k];
        out->com[k] = d[8] != 0.0 ? d[9 + k] / d[8] : 0.0;
    }
    out->mass = d[8];
    return NBODY_OK;
}

int nbody_force_vjp(nbody_ctx *c, uint32_t n, const double *pos, const double *mass, const double *dL_dacc,
                    double *dL_dpos, double *dL_dmass) {
    CTX_OR_FAIL(c);
    if (n > kMaxParticles) return fail(NBODY_ERR_INVALID, "n exceeds the 2^28 particle limit%s");
    if (n && (!pos || !mass || !dL_dacc || !dL_dpos || !dL_dmass)) return fail(NBODY_ERR_INVALID, "null array%s");
    if (single(c)) return fail(NBODY_ERR_INVALID, "the adjoint needs datatype_bytes 8%s");
    if (n == 0) return NBODY_OK;
    int rc = upload(c, n, pos, nullptr, mass);
    if (rc) return rc;
    c->have_fwd = false;  // the state and the adjoint buffers are reused here
    if ((rc = reserve_adjoint(c, n, 1, 0))) return rc;
    if ((rc = begin_call(c))) return rc;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    NB_CUDA(cudaMemcpyAsync(c->lx, dL_dacc, 24 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if (fp64) {
        NB_CUDA(cudaMemcpyAsync(c->lam, c->lx, 24 * (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        NB_CUDA(launch_lam_to_float_scaled(c->lx, (float *)c->lam, 3 * (size_t)n, c->sc, c->stream));
        c->launches += 2;
    }
    NB_CUDA(cudaMemsetAsync(c->lx, 0, 24 * (size_t)n, c->stream));
    NB_CUDA(cudaMemsetAsync(c->lm, 0, 8 * (size_t)n, c->stream));
    if ((rc = adjoint_force(c, c->pos, c->p.damping, c->p.theta, fp64))) return rc;
    NB_CUDA(cudaMemcpyAsync(dL_dpos, c->lx, 24 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaMemcpyAsync(dL_dmass, c->lm, 8 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_forward_checkpointed(nbody_ctx *c, uint32_t nsteps, uint32_t every) {
    CTX_OR_FAIL(c);
    if (!c->have_state || !c->have_vel) return fail(NBODY_ERR_STATE, "particles with velocities must be set first%s");
    if (c->p.adaptive) return fail(NBODY_ERR_INVALID, "the adjoint needs a fixed dt (adaptive = 0)%s");
    if (merging(c)) return fail(NBODY_ERR_INVALID, "the adjoint cannot differentiate through merging%s");
    if (single(c)) return fail(NBODY_ERR_INVALID, "the adjoint needs datatype_bytes 8%s");
    c->have_fwd = false;
    if (nsteps == 0 || c->n == 0) return NBODY_OK;
    MultiStepCall scope(c, nsteps > 1);
    if (every == 0) {
        every = 1;
        while ((uint64_t)every * every < nsteps) every++;
    }
    if (every > nsteps) every = nsteps;
    const uint32_t nseg = (nsteps + every - 1) / every;
    int rc = reserve_adjoint(c, c->n, every, nseg, true);
    if (rc) return rc;
    if ((rc = begin_call(c))) return rc;
    if ((rc = maybe_autotune(c))) return rc;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    const size_t N3 = 3 * (size_t)c->n;
    (void)fp64;
    for (uint32_t k = 0; k < nsteps; k += every) {
        double *ck = c->ckpt + 2 * N3 * (k / every);
        NB_CUDA(cudaMemcpyAsync(ck, c->pos, 8 * N3, cudaMemcpyDeviceToDevice, c->stream));
        NB_CUDA(cudaMemcpyAsync(ck + N3, c->vel, 8 * N3, cudaMemcpyDeviceToDevice, c->stream));
        const uint32_t len = nsteps - k < every ? nsteps - k : every;
        if ((rc = run_steps(c, len))) return rc;
    }
    if ((rc = copy_scalars_back(c))) return rc;
    if ((rc = check_status(c))) return rc;
    c->fwd_steps = nsteps;
    c->fwd_every = every;
    c->fwd_n = c->n;
    c->fwd_dt = c->p.dt;
    c->have_fwd = true;
    return NBODY_OK;
}

int nbody_backward(nbody_ctx *c, const double *dL_dpos, const double *dL_dvel, double *dL_dpos0, double *dL_dvel0,
                   double *dL_dmass) {
    CTX_OR_FAIL(c);
    if (!c->have_fwd || c->fwd_n != c->n) return fail(NBODY_ERR_STATE, "call nbody_forward_checkpointed first%s");
    if (!dL_dpos || !dL_dpos0 || !dL_dvel0 || !dL_dmass) return fail(NBODY_ERR_INVALID, "null array%s");
    const uint32_t n = c->n, K = c->fwd_steps, C = c->fwd_every;
    const size_t N3 = 3 * (size_t)n;
    const bool fp64 = c->p.precision == NBODY_PRECISION_FP64;
    if (c->p.dt != c->fwd_dt) return fail(NBODY_ERR_STATE, "dt changed since the forward pass%s");
    MultiStepCall scope(c, K > 1);
    int rc = begin_call(c);
    if (rc) return rc;
    {
        auto key = graph_key(c, C);
        if (key != c->adj_key) {
            for (auto &g : c->rec_exec) drop_graph(g);
            for (auto &g : c->adj_exec) drop_graph(g);
            c->rec_exec.clear(); c->adj_exec.clear();
            c->rec_launches.clear(); c->adj_launches.clear();
            c->adj_key = key;
        }
    }
    NB_CUDA(cudaMemcpyAsync(c->lx, dL_dpos, 8 * N3, cudaMemcpyHostToDevice, c->stream));
    if (dL_dvel) NB_CUDA(cudaMemcpyAsync(c->lv, dL_dvel, 8 * N3, cudaMemcpyHostToDevice, c->stream));
    else NB_CUDA(cudaMemsetAsync(c->lv, 0, 8 * N3, c->stream));
    NB_CUDA(cudaMemsetAsync(c->lm, 0, 8 * (size_t)n, c->stream));
    const uint32_t nseg = (K + C - 1) / C;
    for (int seg = (int)nseg - 1; seg >= 0; seg--) {
        const uint32_t k0 = (uint32_t)seg * C, len = (K - k0 < C) ? K - k0 : C;
        const double *ck = c->ckpt + 2 * N3 * (size_t)seg;
        NB_CUDA(cudaMemcpyAsync(c->seg_pos, ck, 8 * N3, cudaMemcpyDeviceToDevice, c->stream));
        NB_CUDA(cudaMemcpyAsync(c->vel_work, ck + N3, 8 * N3, cudaMemcpyDeviceToDevice, c->stream));
        for (uint32_t i = 0; i + 1 < len; i++) {
            auto rec = [&, i]() -> int {
                double *xi = c->seg_pos + N3 * i, *xn = xi + N3;
                NB_CUDA(cudaMemcpyAsync(xn, xi, 8 * N3, cudaMemcpyDeviceToDevice, c->stream));
                // forces at xi, then update the copy in place: x_{k+1}, v_{k+1}
                const int save = i < c->n_slots ? (int)i : -1;
                int r = force_pass(c, c->p.damping, c->p.theta, fp64, false, false, false, false, xi, false, nullptr,
                                   false, save, -1);
                if (r) return r;
                StepParams sp{c->p.dt, 0, 0, 0, 0};
                NB_CUDA(launch_update(xn, c->vel_work, c->acc, fp64, n, sp, c->sc, c->stream));
                c->launches++;
                return NBODY_OK;
            };
            if ((rc = run_cached(c, c->rec_exec, c->rec_launches, i, rec))) return rc;
        }
        for (int i = (int)len - 1; i >= 0; i--) {
            auto adj = [&, i]() -> int {
                if (fp64) {
                    NB_CUDA(launch_adj_pre(c->lx, c->lv, c->lam, c->p.dt, n, c->stream));
                    c->launches++;
                } else {
                    // dL/da in FP64 (gdir is free until the walk), then scaled into FP32
                    double *lam_d = c->gdir;
                    NB_CUDA(launch_adj_pre(c->lx, c->lv, lam_d, c->p.dt, n, c->stream));
                    NB_CUDA(launch_lam_to_float_scaled(lam_d, (float *)c->lam, N3, c->sc, c->stream));
                    c->launches += 3;
                }
                // positions 0 .. len-2 of the segment had their octrees saved by the recomputation
                const int restore = (uint32_t)i + 1 < len && (uint32_t)i < c->n_slots ? i : -1;
                return adjoint_force(c, c->seg_pos + N3 * (size_t)i, c->p.damping, c->p.theta, fp64, restore);
            };
            if ((rc = run_cached(c, c->adj_exec, c->adj_launches, (uint32_t)i, adj))) return rc;
        }
    }
    NB_CUDA(cudaMemcpyAsync(dL_dpos0, c->lx, 8 * N3, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaMemcpyAsync(dL_dvel0, c->lv, 8 * N3, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaMemcpyAsync(dL_dmass, c->lm, 8 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = copy_scalars_back(c))) return rc;
    return check_status(c);
}

int nbody_save_frame(nbody_ctx *c, const char *dir, uint32_t frame, int binary, int text, int datatype_bytes) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (datatype_bytes != 8 && datatype_bytes != 4) return fail(NBODY_ERR_INVALID, "datatype_bytes must be 8 or 4%s");
    const size_t n = c->n;
    std::vector<double> pos(3 * n), vel(3 * n, 0.0), acc(3 * n, 0.0), mass(n);
    int rc = nbody_get_particles(c, pos.data(), c->have_vel ? vel.data() : nullptr, c->have_acc ? acc.data() : nullptr);
    if (rc) return rc;
    NB_CUDA(cudaMemcpyAsync(mass.data(), c->mass, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    char path[4096];
    if (binary) {
        if (nbody_frame_path(dir, frame, 1, path, sizeof path) ||
            nbody_write_dat(path, c->n, pos.data(), vel.data(), acc.data(), mass.data(), datatype_bytes))
            return fail(NBODY_ERR_INVALID, "cannot write binary frame %.400s", path);
    }
    if (text) {
        if (nbody_frame_path(dir, frame, 0, path, sizeof path) ||
            nbody_write_txt(path, c->n, pos.data(), datatype_bytes))
            return fail(NBODY_ERR_INVALID, "cannot write text frame %.400s", path);
    }
    return NBODY_OK;
}

int nbody_load_frame(nbody_ctx *c, const char *dir, uint32_t num_frames, int datatype_bytes, uint32_t *next_frame) {
    CTX_OR_FAIL(c);
    if (!next_frame) return fail(NBODY_ERR_INVALID, "next_frame is null%s");
    int32_t f = -1;
    if (nbody_find_resume_frame(dir, num_frames, &f)) return fail(NBODY_ERR_INVALID, "bad frame directory%s");
    if (f < 0) {  // nothing to resume: read_data returns 0 and the caller generates
        *next_frame = 0;
        return NBODY_OK;
    }
    char path[4096];
    uint32_t n = 0;
    if (nbody_frame_path(dir, (uint32_t)f, 1, path, sizeof path) ||
        nbody_read_dat(path, datatype_bytes, &n, nullptr, nullptr, nullptr, nullptr))
        return fail(NBODY_ERR_INVALID, "cannot read %.400s", path);
    std::vector<double> pos(3 * (size_t)n), vel(3 * (size_t)n), mass(n);
    if (nbody_read_dat(path, datatype_bytes, &n, pos.data(), vel.data(), nullptr, mass.data()))
        return fail(NBODY_ERR_INVALID, "cannot read %.400s", path);
    int rc = nbody_set_particles(c, n, pos.data(), vel.data(), mass.data());
    if (rc) return rc;
    *next_frame = (uint32_t)f + 1;
    return NBODY_OK;
}

int nbody_direct_forces(nbody_ctx *c, uint32_t m, const uint32_t *targets, int damping, double *acc_out) {
    CTX_OR_FAIL(c);
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    if (m && !acc_out) return fail(NBODY_ERR_INVALID, "acc_out is null%s");
    if (!targets && m > c->n) return fail(NBODY_ERR_INVALID, "m exceeds the particle count%s");
    if (targets)
        for (uint32_t w = 0; w < m; w++)
            if (targets[w] >= c->n) return fail(NBODY_ERR_INVALID, "target index out of range%s");
    if (m == 0) return NBODY_OK;
    const size_t need = align256(4 * (size_t)m) + align256(24 * (size_t)m);
    if (need > c->direct_bytes) {
        NB_CUDA(cudaStreamSynchronize(c->stream));
        if (c->direct_arena) NB_CUDA(cudaFree(c->direct_arena));
        c->direct_arena = nullptr;
        c->direct_bytes = 0;
        cudaError_t e = cudaMalloc(&c->direct_arena, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(NBODY_ERR_OOM, "direct-sum buffers (%s)", cudaGetErrorString(e));
        }
        c->direct_bytes = need;
    }
    uint32_t *d_t = (uint32_t *)c->direct_arena;
    double *d_out = (double *)((char *)c->direct_arena + align256(4 * (size_t)m));
    if (targets) NB_CUDA(cudaMemcpyAsync(d_t, targets, 4 * (size_t)m, cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(launch_direct(c->pos, c->mass, c->n, damping, targets ? d_t : nullptr, m, d_out, c->stream));
    c->launches++;
    NB_CUDA(cudaMemcpyAsync(acc_out, d_out, 24 * (size_t)m, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NBODY_OK;
}

void nbody_default_image_params(nbody_image_params *p) {
    if (!p) return;
    p->width = 1920;        // img_w, src/main.cpp:1347
    p->height = 1080;       // img_h, src/main.cpp:1348
    p->projection = 3;      // iso, src/main.cpp:1346
    p->color = 0;           // bw, src/main.cpp:1350
    p->adaptive = 0;        // adaptive_brightness, src/main.cpp:1351
    p->nonlinear = 0;       // nonlinear_brightness, src/main.cpp:1352
    p->scale = 1.0;         // scale, src/main.cpp:1349
    p->brightness = 255.0;  // brightness, src/main.cpp:1345
}

int nbody_render(nbody_ctx *c, const nbody_image_params *ip, uint8_t *rgb_out) {
    CTX_OR_FAIL(c);
    if (!ip || !rgb_out || ip->width == 0 || ip->height == 0 || ip->projection < 0 || ip->projection > 3 ||
        ip->color < 0 || ip->color > 1 || (uint64_t)ip->width * ip->height > (1ull << 28))
        return fail(NBODY_ERR_INVALID, "invalid image parameters%s");
    if (!c->have_state) return fail(NBODY_ERR_STATE, "no particles set%s");
    const size_t pixels = (size_t)ip->width * ip->height;
    const size_t need = align256(8 * pixels) + align256(8) + align256(3 * pixels);
    if (need > c->img_bytes) {
        NB_CUDA(cudaStreamSynchronize(c->stream));
        if (c->img_arena) NB_CUDA(cudaFree(c->img_arena));
        c->img_arena = nullptr;
        c->img_bytes = 0;
        cudaError_t e = cudaMalloc(&c->img_arena, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(NBODY_ERR_OOM, "image buffers (%s)", cudaGetErrorString(e));
        }
        c->img_bytes = need;
    }
    char *p = (char *)c->img_arena;
    double *grid = (double *)p;
    unsigned long long *maxbits = (unsigned long long *)(p + align256(8 * pixels));
    uint8_t *rgb = (uint8_t *)(p + align256(8 * pixels) + align256(8));
    ImageArgs a{ip->width, ip->height, ip->projection, ip->color, ip->adaptive, ip->nonlinear, ip->scale,
                ip->brightness};
    NB_CUDA(render_image(c->pos, c->n, a, grid, maxbits, rgb, c->stream));
    c->launches += 3;
    NB_CUDA(cudaMemcpyAsync(rgb_out, rgb, 3 * pixels, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(cudaStreamSynchronize(c->stream));
    return NBODY_OK;
}

const char *nbody_status_string(int s) {
    switch (s) {
        case NBODY_OK: return "ok";
        case NBODY_ERR_INVALID: return "invalid argument";
        case NBODY_ERR_CUDA: return "CUDA error";
        case NBODY_ERR_OOM: return "out of memory";
        case NBODY_ERR_COINCIDENT: return "coincident particles";
        case NBODY_ERR_NONFINITE: return "non-finite position or mass";
        case NBODY_ERR_CAPACITY: return "walk stack capacity exceeded";
        case NBODY_ERR_NO_DEVICE: return "no sm_100 CUDA device";
        case NBODY_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

const char *nbody_last_error_message(void) { return g_msg; }

}  // extern "C"
