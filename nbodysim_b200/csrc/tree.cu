// Octree construction on the GPU: root cube, Morton-order keys, radix sort,
// binary radix tree, chain-free octree, bottom-up mass / centre of mass.
//
// The tree is the reference's octree (src/octree.cpp:54-196, src/main.cpp:887-927)
// with single-child chains collapsed: a node exists here iff the reference
// node at the same cell has two or more non-empty children (or is the root's
// first branching descendant). Chains carry the same mass and, up to rounding
// emulated below, the same centre of mass as their bottom node, so every
// particle's walk accepts the same bodies (see walk.cu).
#include "tree.cuh"
#include "sort.cuh"

#include <cstdio>

namespace nbody {

// ---------------------------------------------------------------------------
// Root cube from the extrema: bbox midpoint; side = largest extent + 2.0, a tie
// for the largest extent falls through to the z extent (src/main.cpp:898-920).
// The FLOAT build computes it from float extrema (the extrema of the rounded
// positions are the rounded extrema): center = float(lo + hi) / 2.0 rounded to
// float, extents in float, side = float(extent + 2.0).
__device__ inline void root_from_extrema(const double *lo, const double *hi, bool single, double *center,
                                         double *side) {
    if (single) {
        float l[3], h[3];
        for (int k = 0; k < 3; k++) {
            l[k] = __double2float_rn(lo[k]);
            h[k] = __double2float_rn(hi[k]);
            center[k] = (double)__double2float_rn(__dmul_rn((double)__fadd_rn(l[k], h[k]), 0.5));
        }
        const float ex = __fsub_rn(h[0], l[0]), ey = __fsub_rn(h[1], l[1]), ez = __fsub_rn(h[2], l[2]);
        float e;
        if (ex > ey && ex > ez) e = ex;
        else if (ey > ex && ey > ez) e = ey;
        else e = ez;
        *side = (double)__double2float_rn(__dadd_rn((double)e, 2.0));
        return;
    }
    for (int k = 0; k < 3; k++) center[k] = (lo[k] + hi[k]) / 2.0;
    const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    if (ex > ey && ex > ez) *side = ex + 2.0;
    else if (ey > ex && ey > ez) *side = ey + 2.0;
    else *side = ez + 2.0;
}

// Root cube (root_from_extrema) over all particles. Also flags
// non-finite positions (masses are checked where the bodies are gathered), and
// (optionally) reduces max |v| for the adaptive step.
__global__ void k_bbox(const double *__restrict__ pos, const double *__restrict__ vel, uint32_t n,
                       double *__restrict__ partial, DevScalars *sc, int keep_root, int single) {
    griddep();
    __shared__ double s_red[7][32];
    __shared__ bool s_last;
    double mn[3] = {INFINITY, INFINITY, INFINITY};
    double mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    double vmax = 0.0;
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
        bad |= !(isfinite(x) && isfinite(y) && isfinite(z));
        mn[0] = fmin(mn[0], x); mx[0] = fmax(mx[0], x);
        mn[1] = fmin(mn[1], y); mx[1] = fmax(mx[1], y);
        mn[2] = fmin(mn[2], z); mx[2] = fmax(mx[2], z);
        if (vel) {
            double vx = vel[3 * (size_t)i], vy = vel[3 * (size_t)i + 1], vz = vel[3 * (size_t)i + 2];
            vmax = fmax(vmax, vx * vx + vy * vy + vz * vz);  // |v|^2; the square root of the maximum at the end
        }
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&sc->status, kStatusNonFinite);
    double v[7] = {mn[0], mn[1], mn[2], -mx[0], -mx[1], -mx[2], -vmax};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = 0; k < 7; k++) {
        double r = warp_min(v[k]);
        if (lane == 0) s_red[k][wid] = r;
    }
    __syncthreads();
    if (wid == 0) {
        for (int k = 0; k < 7; k++) {
            double r = lane < nw ? s_red[k][lane] : INFINITY;
            r = warp_min(r);
            if (lane == 0) partial[7 * blockIdx.x + k] = r;
        }
        if (lane == 0) {
            __threadfence();
            s_last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!s_last) return;
    // The last block reduces every block's partials: each thread takes whole
    // rows (seven independent loads), then a block reduction.
    __threadfence();
    double acc[7];
#pragma unroll
    for (int k = 0; k < 7; k++) acc[k] = INFINITY;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 7; k++) acc[k] = fmin(acc[k], __ldcg(&partial[7 * b + k]));
    }
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double m = warp_min(acc[k]);
        if (lane == 0) s_red[k][wid] = m;
    }
    __syncthreads();
    if (wid != 0) return;
    double r[7];
#pragma unroll
    for (int k = 0; k < 7; k++) r[k] = warp_min(lane < nw ? s_red[k][lane] : INFINITY);
    if (lane == 0 && keep_root) {
        sc->max_vel_bits = (unsigned long long)__double_as_longlong(sqrt(-r[6]));
        sc->ticket = 0;
    } else if (lane == 0) {
        double lo[3] = {r[0], r[1], r[2]}, hi[3] = {-r[3], -r[4], -r[5]};
        for (int k = 0; k < 3; k++) {
            sc->bbox_min[k] = lo[k];
            sc->bbox_max[k] = hi[k];
        }
        double center[3], side;
        root_from_extrema(lo, hi, single != 0, center, &side);
        for (int k = 0; k < 3; k++) sc->root_center[k] = center[k];
        sc->root_side = side;
        sc->max_vel_bits = (unsigned long long)__double_as_longlong(sqrt(-r[6]));
        sc->ticket = 0;
    }
}

// Root cube per system (several independent systems): one block per system.
__global__ void k_bbox_systems(const double *__restrict__ pos, const double *__restrict__ mass,
                               const uint32_t *__restrict__ sys_start, double *__restrict__ sys_root,
                               DevScalars *sc, int single) {
    griddep();
    __shared__ double s_red[6][32];
    const uint32_t b0 = sys_start[blockIdx.x], b1 = sys_start[blockIdx.x + 1];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool bad = false;
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
        bad |= !(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(mass[i]));
        mn[0] = fmin(mn[0], x); mx[0] = fmax(mx[0], x);
        mn[1] = fmin(mn[1], y); mx[1] = fmax(mx[1], y);
        mn[2] = fmin(mn[2], z); mx[2] = fmax(mx[2], z);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&sc->status, kStatusNonFinite);
    double v[6] = {mn[0], mn[1], mn[2], -mx[0], -mx[1], -mx[2]};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = 0; k < 6; k++) {
        const double r = warp_min(v[k]);
        if (lane == 0) s_red[k][wid] = r;
    }
    __syncthreads();
    if (wid != 0) return;
    double r[6];
    for (int k = 0; k < 6; k++) r[k] = warp_min(lane < nw ? s_red[k][lane] : INFINITY);
    if (lane == 0) {
        const double lo[3] = {r[0], r[1], r[2]}, hi[3] = {-r[3], -r[4], -r[5]};
        double *o = sys_root + 4 * (size_t)blockIdx.x;
        root_from_extrema(lo, hi, single != 0, o, o + 3);
    }
}

// ---------------------------------------------------------------------------
// Octant digits by descent from the root cube, rounding every child centre
// exactly as allocate_child does (src/octree.cpp:65-84: center + (+-1 * half) / 2
// with half = side / 2), and choosing the octant with strict '>' as
// add_particle does (src/octree.cpp:153-165). Digits are (z<<2)|(y<<1)|x so
// that Morton order equals the reference's child order 0..7. T is the
// reference build's datatype: double, or float for its FLOAT build.
__device__ inline double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ inline float add_rn(float a, float b) { return __fadd_rn(a, b); }

template <typename T>
__device__ inline uint64_t descend_word(T x, T y, T z, T &cx, T &cy, T &cz, T &side) {
    uint64_t key = 0;
#pragma unroll 3
    for (int l = 0; l < kLevelsPerWord; l++) {
        const T half = side / T(2);
        const T q = half / T(2);
        int bx = x > cx, by = y > cy, bz = z > cz;
        key = (key << 3) | (uint64_t)((bz << 2) | (by << 1) | bx);
        cx = add_rn(cx, bx ? q : -q);
        cy = add_rn(cy, by ? q : -q);
        cz = add_rn(cz, bz ? q : -q);
        side = half;
    }
    return key;
}

// `words` key words of one particle from the root cube (center, side).
template <typename T>
__device__ inline void descend_words(const double *p, const double *root, int words, uint64_t *out) {
    T cx = (T)root[0], cy = (T)root[1], cz = (T)root[2], s = (T)root[3];
    const T x = (T)p[0], y = (T)p[1], z = (T)p[2];
    for (int w = 0; w < words; w++) out[w] = descend_word<T>(x, y, z, cx, cy, cz, s);
}

// Key words per particle: levels 1..21 (k1) and 22..42 (k2). Escaped
// particles can make the root cube many orders of magnitude larger than the
// bulk of the system, so the first 21 levels alone do not separate it. With
// k2_user null only k1 is computed (a sort plan that needs no second word).
// The sort key (k1 or k2) goes to `sortkey`, the identity to `idx`.
__global__ void k_keys(const double *__restrict__ pos, uint32_t n, const DevScalars *sc,
                       uint64_t *__restrict__ k1_user, uint64_t *__restrict__ sortkey,
                       uint64_t *__restrict__ k2_user, uint32_t *__restrict__ idx,
                       const uint32_t *__restrict__ sys_id, const double *__restrict__ sys_root, int single,
                       int sort_by_k1) {
    griddep();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double root[4];
    if (sys_id) {
        const double *r = sys_root + 4 * (size_t)sys_id[i];
        root[0] = r[0]; root[1] = r[1]; root[2] = r[2]; root[3] = r[3];
    } else {
        root[0] = sc->root_center[0]; root[1] = sc->root_center[1]; root[2] = sc->root_center[2];
        root[3] = sc->root_side;
    }
    const double p[3] = {pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2]};
    const int words = k2_user ? 2 : 1;
    uint64_t w[2] = {0, 0};
    if (single) descend_words<float>(p, root, words, w);
    else descend_words<double>(p, root, words, w);
    k1_user[i] = w[0];
    sortkey[i] = sort_by_k1 ? w[0] : w[1];
    if (k2_user) k2_user[i] = w[1];
    idx[i] = i;
}

// The second key words (single system), for a full sort that follows a plan
// without them; nothing unless *run_if is non-zero.
__global__ void k_keys_second(const double *__restrict__ pos, uint32_t n, const DevScalars *sc,
                              uint64_t *__restrict__ k2_user, int single, const uint32_t *run_if) {
    griddep();
    if (*run_if == 0u) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double root[4] = {sc->root_center[0], sc->root_center[1], sc->root_center[2], sc->root_side};
    const double p[3] = {pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2]};
    uint64_t w[2];
    if (single) descend_words<float>(p, root, 2, w);
    else descend_words<double>(p, root, 2, w);
    k2_user[i] = w[1];
}

// dst[j] = src[idx[j]]; with run_if non-null, only when *run_if is non-zero.
__global__ void k_gather_key(const uint64_t *__restrict__ src, const uint32_t *__restrict__ idx,
                             uint64_t *__restrict__ dst, uint32_t n, const uint32_t *run_if) {
    griddep();
    if (run_if && *run_if == 0u) return;
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) dst[j] = src[idx[j]];
}

// Runs of neighbours that the sort plan left equal over its bits, (k1 >> s1)
// and, when the plan sorted part of the second word, (k2 >> s2), are put in
// order here: each run of at most kMaxTieRun particles is sorted in place by
// the full keys (k1, then k2; k2 in key_a, computed here for the run when the
// plan had no second words), with a stable insertion sort, so that equal keys
// keep the user order as the full LSD sort keeps it. Runs are disjoint and a
// permutation inside a run leaves every prefix of the run unchanged, so the
// runs are found and sorted concurrently. A longer run sets the flag of the
// full sort (inside a captured graph, the condition of its graph node).
constexpr uint32_t kMaxTieRun = 64;

__global__ void k_fix_ties(uint64_t *__restrict__ k1_sorted, uint64_t *__restrict__ k2_sorted,
                           uint32_t *__restrict__ idx, const double *__restrict__ pos, int have_k2, int s1, int s2,
                           uint32_t n, int single, DevScalars *sc, cudaGraphConditionalHandle cond, int use_cond) {
    griddep();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    auto same = [&](uint32_t a, uint32_t b) {
        bool t = (k1_sorted[a] >> s1) == (k1_sorted[b] >> s1);
        if (t && have_k2) t = (k2_sorted[a] >> s2) == (k2_sorted[b] >> s2);
        return t;
    };
    if (j + 1 >= n || !same(j, j + 1) || (j > 0 && same(j - 1, j))) return;  // not the first of a run
    uint32_t e = j + 1;
    while (e + 1 < n && same(e, e + 1)) {
        if (++e - j + 1 > kMaxTieRun) {
            atomicOr(&sc->word_ties, 1u);
            if (use_cond) cudaGraphSetConditional(cond, 1u);
            return;
        }
    }
    atomicAdd(&sc->tie_runs, 1u);
    if (!have_k2) {
        // The plan sorted top bits of the first word only: the run is sorted by its
        // first words, and only a stretch of equal first words needs the second
        // word, computed for it here (stable sorts both, as the full sort is).
        for (uint32_t q = j + 1; q <= e; q++) {
            const uint64_t a1 = k1_sorted[q];
            const uint32_t ai = idx[q];
            uint32_t p = q;
            while (p > j && k1_sorted[p - 1] > a1) {
                k1_sorted[p] = k1_sorted[p - 1];
                idx[p] = idx[p - 1];
                p--;
            }
            k1_sorted[p] = a1;
            idx[p] = ai;
        }
        const double root[4] = {sc->root_center[0], sc->root_center[1], sc->root_center[2], sc->root_side};
        for (uint32_t a = j; a < e;) {
            uint32_t b = a;
            while (b < e && k1_sorted[b + 1] == k1_sorted[a]) b++;
            if (b > a) {
                for (uint32_t q = a; q <= b; q++) {
                    const size_t u = 3 * (size_t)idx[q];
                    const double p[3] = {pos[u], pos[u + 1], pos[u + 2]};
                    uint64_t w[2];
                    if (single) descend_words<float>(p, root, 2, w);
                    else descend_words<double>(p, root, 2, w);
                    k2_sorted[q] = w[1];
                }
                for (uint32_t q = a + 1; q <= b; q++) {
                    const uint64_t a2 = k2_sorted[q];
                    const uint32_t ai = idx[q];
                    uint32_t p = q;
                    while (p > a && k2_sorted[p - 1] > a2) {
                        k2_sorted[p] = k2_sorted[p - 1];
                        idx[p] = idx[p - 1];
                        p--;
                    }
                    k2_sorted[p] = a2;
                    idx[p] = ai;
                }
            }
            a = b + 1;
        }
        return;
    }
    for (uint32_t q = j + 1; q <= e; q++) {
        const uint64_t a1 = k1_sorted[q], a2 = k2_sorted[q];
        const uint32_t ai = idx[q];
        uint32_t p = q;
        while (p > j && (k1_sorted[p - 1] > a1 || (k1_sorted[p - 1] == a1 && k2_sorted[p - 1] > a2))) {
            k1_sorted[p] = k1_sorted[p - 1];
            k2_sorted[p] = k2_sorted[p - 1];
            idx[p] = idx[p - 1];
            p--;
        }
        k1_sorted[p] = a1;
        k2_sorted[p] = a2;
        idx[p] = ai;
    }
}

// Start of the full sort after ties: the second words as sort keys, identity indices.
__global__ void k_full_sort_init(const uint64_t *__restrict__ k2_user, uint64_t *__restrict__ key,
                                 uint32_t *__restrict__ idx, uint32_t n, const uint32_t *run_if) {
    griddep();
    if (*run_if == 0u) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        key[i] = k2_user[i];
        idx[i] = i;
    }
}

__global__ void k_gather_sys(const uint32_t *__restrict__ sys_id, const uint32_t *__restrict__ idx,
                             uint64_t *__restrict__ key, uint32_t *__restrict__ sys_sorted, uint32_t n) {
    griddep();
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t s = sys_id[idx[j]];
    if (key) key[j] = s;
    if (sys_sorted) sys_sorted[j] = s;
}

// Exclusive prefix sum of u32 values in place: tiles of 4096 scanned per
// block, tile totals scanned by one block, then added back.
constexpr int kScanThreads = 1024;
constexpr int kScanTile = 4 * kScanThreads;

__device__ inline uint32_t block_exclusive_scan(uint32_t x, uint32_t *s_warp, uint32_t *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
        uint32_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        s_warp[lane] = wi - w;
        if (lane == 31) s_warp[32] = wi;
    }
    __syncthreads();
    uint32_t r = s_warp[wid] + incl - x;
    if (total) *total = s_warp[32];
    return r;
}

__global__ void k_scan_tiles(uint32_t *__restrict__ v, uint32_t len, uint32_t *__restrict__ tile_sums) {
    griddep();
    __shared__ uint32_t s_warp[33];
    const uint32_t base = blockIdx.x * kScanTile + 4 * threadIdx.x;
    uint32_t x[4];
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = base + k < len ? v[base + k] : 0u;
    uint32_t s = x[0] + x[1] + x[2] + x[3];
    uint32_t tot;
    uint32_t run = block_exclusive_scan(s, s_warp, &tot);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (base + k < len) v[base + k] = run;
        run += x[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// One block: exclusive scan of up to a few thousand tile totals; writes the grand total.
__global__ void k_scan_small(uint32_t *__restrict__ v, uint32_t len, uint32_t *total) {
    griddep();
    __shared__ uint32_t s_warp[33];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < len; b += blockDim.x) {
        uint32_t i = b + threadIdx.x;
        uint32_t x = i < len ? v[i] : 0u;
        uint32_t tot;
        uint32_t r = block_exclusive_scan(x, s_warp, &tot);
        if (i < len) v[i] = r + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_add(uint32_t *__restrict__ v, uint32_t len, const uint32_t *__restrict__ tile_sums) {
    griddep();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < len) v[i] += tile_sums[i / kScanTile];
}

unsigned scan_exclusive(uint32_t *v, uint32_t len, uint32_t *tile_sums, uint32_t *total, cudaStream_t st) {
    const uint32_t tiles = (len + kScanTile - 1) / kScanTile;
    launch_pdl(k_scan_tiles, dim3(tiles), dim3(kScanThreads), 0, st, v, len, tile_sums);
    launch_pdl(k_scan_small, dim3(1), dim3(kScanThreads), 0, st, tile_sums, tiles, total);
    if (tiles > 1) launch_pdl(k_scan_add, dim3((len + 255) / 256), dim3(256), 0, st, v, len, tile_sums);
    return tiles > 1 ? 3u : 2u;
}

// ---------------------------------------------------------------------------
// Bodies in sorted order (as floats in the FLOAT build); flags non-finite masses.
__global__ void k_gather_bodies(const uint32_t *__restrict__ idx, const double *__restrict__ pos,
                                const double *__restrict__ mass, double4 *__restrict__ body,
                                uint32_t n, DevScalars *sc, int single) {
    griddep();
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t i = idx[j];
    double m = mass[i];
    if (!isfinite(m)) atomicOr(&sc->status, kStatusNonFinite);
    double4 b = make_double4(pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], m);
    if (single) {
        b.x = (double)__double2float_rn(b.x); b.y = (double)__double2float_rn(b.y);
        b.z = (double)__double2float_rn(b.z); b.w = (double)__double2float_rn(b.w);
    }
    body[j] = b;
}

// Groups of particles whose 42-level keys agree get a third key word (levels
// 43..63) and are re-sorted among themselves. Identical keys over all 63
// levels mean coincident particles (the reference recurses without bound).
constexpr int kMaxDeepGroup = 64;

__global__ void k_deep_groups(const uint64_t *__restrict__ key1, const uint64_t *__restrict__ key2,
                              uint64_t *__restrict__ key3, uint32_t *__restrict__ idx,
                              double4 *__restrict__ body, uint32_t n, const uint32_t *__restrict__ sys,
                              const double *__restrict__ sys_root, DevScalars *sc, int single) {
    griddep();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= n) return;
    const uint64_t k = key1[i], kk = key2[i];
    const uint32_t ss = sys ? sys[i] : 0u;
    auto same = [&](uint32_t q) { return key1[q] == k && key2[q] == kk && (!sys || sys[q] == ss); };
    if (!same(i + 1)) return;
    if (i > 0 && same(i - 1)) return;  // not the first of its group
    uint32_t e = i + 1;
    while (e + 1 < n && same(e + 1)) e++;
    const uint32_t g = e - i + 1;
    atomicAdd(&sc->deep_groups, 1u);
    atomicOr(&sc->status, kStatusDeepGroup);
    if (g > kMaxDeepGroup) {
        // More than 64 particles inside one cell of side 2^-42 of the root:
        // reported as coincident. Zero third words keep the radix tree well
        // formed (ties then break on sorted position).
        for (uint32_t j = i; j <= e; j++) key3[j] = 0;
        atomicOr(&sc->status, kStatusCoincident);
        return;
    }
    double root[4] = {sc->root_center[0], sc->root_center[1], sc->root_center[2], sc->root_side};
    if (sys) {
        const double *r = sys_root + 4 * (size_t)ss;
        root[0] = r[0]; root[1] = r[1]; root[2] = r[2]; root[3] = r[3];
    }
    for (uint32_t j = i; j <= e; j++) {
        const double4 b = body[j];
        const double p[3] = {b.x, b.y, b.z};
        uint64_t w[3];
        if (single) descend_words<float>(p, root, 3, w);
        else descend_words<double>(p, root, 3, w);
        key3[j] = w[2];
    }
    // insertion sort of the group by its third word
    for (uint32_t j = i + 1; j <= e; j++) {
        const uint64_t a3 = key3[j];
        const uint32_t ai = idx[j];
        const double4 ab = body[j];
        uint32_t p = j;
        while (p > i && key3[p - 1] > a3) {
            key3[p] = key3[p - 1]; idx[p] = idx[p - 1]; body[p] = body[p - 1];
            p--;
        }
        key3[p] = a3; idx[p] = ai; body[p] = ab;
    }
    for (uint32_t j = i; j < e; j++)
        if (key3[j] == key3[j + 1]) atomicOr(&sc->status, kStatusCoincident);
}

// ---------------------------------------------------------------------------
// Binary radix tree (Karras 2012, "Maximizing parallelism in the construction
// of BVHs, octrees and k-d trees"), prefix lengths in key bits over up to
// three 63-bit words; exact duplicates fall back to index bits so the tree
// stays well formed while the coincident status reports the error.
struct KeyView {
    const uint64_t *k1, *k2, *k3;
    int n;
    const uint32_t *sys;  // system per sorted position, or null (one system)
    __device__ int delta(int i, int j) const {
        if (j < 0 || j >= n) return -1;
        if (sys && sys[i] != sys[j]) return -1;  // separate systems: separate trees
        uint64_t a = k1[i], b = k1[j];
        if (a != b) return __clzll(a ^ b) - 1;
        a = k2[i]; b = k2[j];
        if (a != b) return 63 + __clzll(a ^ b) - 1;
        a = k3[i]; b = k3[j];
        if (a != b) return 126 + __clzll(a ^ b) - 1;
        return 189 + __clz((unsigned)i ^ (unsigned)j);
    }
};

__device__ inline int level_of(int delta) { return min(delta / 3, kMaxLevels); }

// KeyView::delta(i, j) for one i, with i's first key word and system held in
// registers (the kernel's stores could alias the keys, so the compiler would
// load them again for every call); the deeper words only where first words agree.
struct DeltaFrom {
    const KeyView &kv;
    int i;
    uint64_t a1;
    uint32_t si;
    __device__ DeltaFrom(const KeyView &v, int at) : kv(v), i(at), a1(v.k1[at]), si(v.sys ? v.sys[at] : 0u) {}
    __device__ int operator()(int j) const {
        if (j < 0 || j >= kv.n) return -1;
        if (kv.sys && kv.sys[j] != si) return -1;
        const uint64_t b1 = kv.k1[j];
        if (a1 != b1) return __clzll(a1 ^ b1) - 1;
        return kv.delta(i, j);
    }
};

__global__ void k_radix_tree(KeyView kv, int32_t *__restrict__ bleft, int32_t *__restrict__ bright,
                             int32_t *__restrict__ bparent, int32_t *__restrict__ leaf_bparent,
                             int32_t *__restrict__ bdelta, uint32_t *max_prefix_bits, uint32_t *pair_passes) {
    __shared__ uint32_t hist[kPassBins];
    griddep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = kv.n;
    // the deepest split: key bits that separate every pair of neighbours
    const int dn = i < n - 1 ? DeltaFrom(kv, i)(i + 1) : -1;
    const int wmax = __reduce_max_sync(0xffffffffu, dn);
    if ((threadIdx.x & 31) == 0 && wmax >= 0) atomicMax(max_prefix_bits, (uint32_t)wmax + 1u);
    // the pairs by the sort passes that separate them (the next build's plan):
    // per warp one shared-memory add per distinct pass count, per block one
    // global add per nonzero bin
    if (threadIdx.x < kPassBins) hist[threadIdx.x] = 0u;
    __syncthreads();
    {
        const int bin = dn >= 0 ? passes_for_bits((uint32_t)dn + 1u) : -1;
        const uint32_t same = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && (threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(same));
    }
    __syncthreads();
    if (threadIdx.x < kPassBins && hist[threadIdx.x]) atomicAdd(&pair_passes[threadIdx.x], hist[threadIdx.x]);
    if (i >= n - 1) return;
    // With several systems, the internal nodes of the system [s, e) are s..e-2:
    // the last particle of a system indexes no internal node.
    if (kv.sys && kv.sys[i] != kv.sys[i + 1]) {
        bdelta[i] = -1;
        return;
    }
    const bool seg_root = i == 0 || (kv.sys && kv.sys[i - 1] != kv.sys[i]);
    const DeltaFrom di(kv, i);
    const int dprev = di(i - 1);
    int d = (dn - dprev) >= 0 ? 1 : -1;
    int dmin = d > 0 ? dprev : dn;  // delta(i, i - d)
    int lmax = 2;
    while (di(i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (di(i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = di(j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (di(i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    // children encoded: >= 0 internal binary node, < 0 leaf ~index
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    bleft[i] = left;
    bright[i] = right;
    bdelta[i] = dnode;
    if (left >= 0) bparent[left] = i; else leaf_bparent[~left] = i;
    if (right >= 0) bparent[right] = i; else leaf_bparent[~right] = i;
    if (seg_root) bparent[i] = -1;
}

// A binary node heads an octree node iff it is the root or its parent sits
// at a shallower octree level.
// Also the starting values of the collapse and the COM climb: a copy of the
// flags to be scanned in place (head_id), parents "none" (so that a child the
// collapse could not attach, reported as an error, is never followed) and zero
// arrival counts. One thread per particle (n = m + 1).
__global__ void k_head_flags(const int32_t *__restrict__ bparent, const int32_t *__restrict__ bdelta,
                             uint32_t m, uint32_t *__restrict__ flag, uint32_t *__restrict__ head_id,
                             int32_t *__restrict__ oparent, int32_t *__restrict__ leaf_oparent,
                             uint32_t *__restrict__ ocount) {
    griddep();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    leaf_oparent[i] = -1;
    if (i == m) return;
    oparent[i] = -1;
    ocount[i] = 0u;
    uint32_t f = 0u;  // not an internal node (the last particle of a system)
    if (bdelta[i] >= 0) {
        const int p = bparent[i];
        f = (p < 0 || level_of(bdelta[p]) < level_of(bdelta[i])) ? 1u : 0u;
    }
    flag[i] = f;
    head_id[i] = f;
}

// Octree root of every system: the head of the binary node at the system's
// first particle (none for a system of fewer than two particles).
__global__ void k_sys_roots(const uint32_t *__restrict__ sys_start, const uint32_t *__restrict__ flag,
                            const uint32_t *__restrict__ head_id, uint32_t nsys, int32_t *__restrict__ root_node) {
    griddep();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const uint32_t a = sys_start[s], b = sys_start[s + 1];
    root_node[s] = (b - a >= 2 && flag[a]) ? (int32_t)head_id[a] : -1;
}

// Each head gathers, left to right, the exits of its same-level binary
// subtree: leaves and deeper heads. Left-to-right is Morton order, i.e. the
// reference's child order 0..7.
__global__ void k_collapse(const int32_t *__restrict__ bleft, const int32_t *__restrict__ bright,
                           const int32_t *__restrict__ bdelta, const uint32_t *__restrict__ head_id,
                           const uint32_t *__restrict__ flag, uint32_t m, int32_t *__restrict__ ochild,
                           int32_t *__restrict__ ometa, int32_t *__restrict__ oparent,
                           int32_t *__restrict__ leaf_oparent, DevScalars *sc) {
    griddep();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !flag[i]) return;
    const int id = (int)head_id[i];
    const int L = level_of(bdelta[i]);
    int nch = 0, nint = 0;
    // A child that is no binary node of this octree level becomes a child of
    // the octree node, in order.
    auto emit = [&](int ch) {
        if (nch >= 8) {
            atomicOr(&sc->status, kStatusCapacity);
            return;
        }
        if (ch < 0) {
            ochild[8 * id + nch] = ch;
            leaf_oparent[~ch] = id;
        } else {
            const int cid = (int)head_id[ch];
            ochild[8 * id + nch] = cid;
            oparent[cid] = id;
            nint++;
        }
        nch++;
    };
    auto same_level = [&](int ch) { return ch >= 0 && level_of(bdelta[ch]) == L; };
    if (L >= kMaxLevels) {
        // The capped level (keys equal over every word: coincident particles,
        // reported as such) can nest deeper: an in-order walk with a stack, a
        // frame visiting its left child, then its right child.
        int fnode[8], fstate[8];
        int fs = 1;
        fnode[0] = (int)i;
        fstate[0] = 0;
        while (fs > 0) {
            const int x = fnode[fs - 1];
            if (fstate[fs - 1] == 2) { fs--; continue; }
            const int ch = fstate[fs - 1] == 0 ? bleft[x] : bright[x];
            fstate[fs - 1]++;
            if (same_level(ch)) {
                if (fs < 8) { fnode[fs] = ch; fstate[fs] = 0; fs++; }
                else atomicOr(&sc->status, kStatusCapacity);
            } else {
                emit(ch);
            }
        }
    } else {
        // In-order walk over the same-level binary nodes. Their prefix lengths grow
        // strictly downwards and stay within the level's 3 key bits, so the walk is
        // at most 3 binary nodes deep: unrolled, with nothing in local memory.
        const int c1[2] = {bleft[i], bright[i]};
    #pragma unroll
        for (int a = 0; a < 2; a++) {
            const int x = c1[a];
            if (!same_level(x)) {
                emit(x);
                continue;
            }
            const int c2[2] = {bleft[x], bright[x]};
    #pragma unroll
            for (int b = 0; b < 2; b++) {
                const int y = c2[b];
                if (!same_level(y)) {
                    emit(y);
                    continue;
                }
                const int c3[2] = {bleft[y], bright[y]};
    #pragma unroll
                for (int c = 0; c < 2; c++) {
                    if (same_level(c3[c])) atomicOr(&sc->status, kStatusCapacity);  // deeper than 3: malformed
                    else emit(c3[c]);
                }
            }
        }
    }
    ometa[id] = L | (min(nch, 8) << 8) | (min(nint, 8) << 12);
    if (id == 0) oparent[0] = -1;
    // the deepest level: one atomic per group of converged lanes
    const unsigned am = __activemask();
    const uint32_t lmax = __reduce_max_sync(am, (uint32_t)L);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1)) atomicMax(&sc->depth, lmax);
}

// ---------------------------------------------------------------------------
// Bottom-up mass and centre of mass (src/octree.cpp:203-221, 252-278): the
// climb starts at the nodes whose children are all bodies, and a node is
// computed by the thread of its last node child to finish. Sums run in
// child order with explicit round-to-nearest operations (no FMA contraction),
// as the reference computes them. A child separated from its parent by k
// single-child chain nodes enters with its centre of mass passed k times
// through the chain's (c * m) / m, the value the reference's chain top holds.
__device__ inline double3 load_node_com(const double4 *p, double &m) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldcg(q), b = __ldcg(q + 1);
    m = b.y;
    return make_double3(a.x, a.y, b.x);
}

// Round-to-nearest arithmetic of the reference build's datatype.
__device__ inline double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ inline float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ inline double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ inline float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// One node's mass and centre of mass from its children, in the arithmetic of
// T (double, or float for the reference's FLOAT build).
// The node's child list comes in as c0, c1 (its eight slots).
template <typename T>
__device__ inline double4 node_com(const double4 *__restrict__ body, int4 c0, int4 c1,
                                   const int32_t *__restrict__ ometa, const double4 *onode, int L, int nch) {
    T m = 0, sx = 0, sy = 0, sz = 0;
    for (int k = 0; k < nch; k++) {
        const int4 h = k < 4 ? c0 : c1;  // selects, not an indexed array (which would live in local memory)
        const int c = (k & 2) ? ((k & 1) ? h.w : h.z) : ((k & 1) ? h.y : h.x);
        T cmk, cx, cy, cz;
        if (c < 0) {
            const double4 b = body[~c];
            cmk = (T)b.w;
            cx = (T)b.x; cy = (T)b.y; cz = (T)b.z;
        } else {
            double dm;
            const double3 cc = load_node_com(&onode[c], dm);
            cmk = (T)dm;
            cx = (T)cc.x; cy = (T)cc.y; cz = (T)cc.z;
            const int chain = meta_level(ometa[c]) - L - 1;
            for (int t = 0; t < chain; t++) {
                if (cmk == T(0)) {
                    cx = cy = cz = T(0);
                } else {
                    cx = div_rn(mul_rn(cx, cmk), cmk);
                    cy = div_rn(mul_rn(cy, cmk), cmk);
                    cz = div_rn(mul_rn(cz, cmk), cmk);
                }
            }
        }
        m = add_rn(m, cmk);
        sx = add_rn(sx, mul_rn(cx, cmk));
        sy = add_rn(sy, mul_rn(cy, cmk));
        sz = add_rn(sz, mul_rn(cz, cmk));
    }
    double4 out;
    out.w = (double)m;
    if (m == T(0)) {
        out.x = out.y = out.z = 0.0;
    } else {
        out.x = (double)div_rn(sx, m);
        out.y = (double)div_rn(sy, m);
        out.z = (double)div_rn(sz, m);
    }
    return out;
}

template <typename T>
// (launch bounds: 4 resident blocks of 256 threads, 64 registers)
__global__ void __launch_bounds__(256, 4)
    k_com(const double4 *__restrict__ body, const int32_t *__restrict__ leaf_oparent,
          const int32_t *__restrict__ oparent, const int32_t *__restrict__ ochild,
          const int32_t *__restrict__ ometa, double4 *onode, uint32_t *ocount, uint32_t n, DevScalars *sc) {
    griddep();
    // One thread per node; the climb starts at nodes whose children are all
    // bodies, and a node is computed by the last of its node children to finish.
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n - 1 || q >= sc->n_onodes) return;
    int p = (int)q;
    if (meta_ninternal(ometa[p]) != 0) return;
    // A well-formed tree is at most kMaxLevels + 1 internal levels deep; the
    // bound only guards against a malformed tree after a reported error.
    for (int hops = 0; p >= 0; hops++) {
        if (hops > kMaxLevels + 1 || p >= (int)(n - 1)) {
            atomicOr(&sc->status, kStatusCapacity);
            return;
        }
        // The node's structure is final (the collapse wrote it): its metadata, child
        // list and parent load before the arrival count, so that after it only the
        // children's values remain to be read.
        const int32_t meta = ometa[p];
        const int nch = meta_nchild(meta);
        const int4 *cp = reinterpret_cast<const int4 *>(ochild + 8 * (size_t)p);
        const int4 c0 = __ldg(cp), c1 = __ldg(cp + 1);
        const int up = oparent[p];
        if (hops > 0) {
            // One acquire-release count: it publishes the node this thread wrote on
            // the previous hop, and the last node child to arrive sees every
            // other child's result.
            uint32_t old;
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(&ocount[p]) : "memory");
            if (old != (uint32_t)(meta_ninternal(meta) - 1)) return;
        }
        // The reference sums the masses, then the mass-weighted centres, each in
        // child order; both sums run here in one pass over the children.
        const int L = meta_level(meta);
        const double4 out = node_com<T>(body, c0, c1, ometa, onode, L, nch);
        double2 *q = reinterpret_cast<double2 *>(&onode[p]);
        __stcg(q, make_double2(out.x, out.y));
        __stcg(q + 1, make_double2(out.z, out.w));
        p = up;
    }
}

// ---------------------------------------------------------------------------
static inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

cudaError_t build_octree(const TreeBuild &tb, cudaStream_t st, unsigned *launches) {
    const uint32_t n = tb.n;
    unsigned L = 0;
    if (n == 0) return cudaSuccess;
    const bool multi = tb.nsys > 1;
    // root cube (+ max |v| when requested); one per system when there are several
    launch_pdl(k_bbox, dim3(tb.bbox_blocks), dim3(256), 0, st, tb.pos, tb.vel_for_max, n, tb.bbox_partial, tb.sc,
                                           multi ? 0 : tb.keep_root, tb.single);
    if (multi) {
        if (tb.mass_ready) cudaStreamWaitEvent(st, tb.mass_ready, 0);
        launch_pdl(k_bbox_systems, dim3(tb.nsys), dim3(256), 0, st, tb.pos, tb.mass, tb.sys_start, tb.sys_root, tb.sc, tb.single);
        L += 1;
    }
    uint32_t *sort_err = &tb.sc->status;
    uint32_t *ties = &tb.sc->word_ties;
    // `count` LSD passes with the digits of a `plan`-pass sort of one word
    // (digit_shift), histogram and status slots from `slot`, ping-ponging
    // (kin, iin) and (kout, iout): an even count leaves the result in (kin, iin),
    // an odd one in (kout, iout).
    auto passes = [&](uint64_t *kin, uint64_t *kout, uint32_t *iin, uint32_t *iout, int count, int plan, int slot,
                      const uint32_t *run_if, cudaStream_t s) {
        for (int q = 0; q < count; q++) {
            sort_pass(kin, iin, kout, iout, n, slot + q, digit_shift(plan, q), tb.sort_scratch, sort_err,
                      kStatusSortStall, run_if, s, &L);
            uint64_t *tk = kin; kin = kout; kout = tk;
            uint32_t *ti = iin; iin = iout; iout = ti;
        }
    };
    auto gather = [&](const uint64_t *src, uint64_t *dst, const uint32_t *run_if, cudaStream_t s) {
        launch_pdl(k_gather_key, dim3(blocks_for(n, 256)), dim3(256), 0, s, src, tb.idx_a, dst, n, run_if);
        L += 1;
    };
    // Slots: passes on k2 0-7, on k1 8-15, on the system id 16-17; the full sort
    // after a plan that left ties, k2 18-25 and k1 26-33.
    // Every plan leaves k1 in sorted order in key_b and the permutation in idx_a
    // (a plan with an odd pass count starts in the other buffers). The user-order
    // words: k1 in key3, k2 in key2.
    const int p2 = multi ? 8 : tb.sort_p2, p1 = multi ? 8 : tb.sort_p1;
    const bool checked = !multi && tb.sort_checked && !(p2 >= 8 && p1 >= 8);
    if (p2 > 0) {
        uint64_t *k0 = (p2 & 1) ? tb.key_b : tb.key_a, *k0o = (p2 & 1) ? tb.key_a : tb.key_b;
        uint32_t *i0 = (p2 & 1) ? tb.idx_b : tb.idx_a, *i0o = (p2 & 1) ? tb.idx_a : tb.idx_b;
        launch_pdl(k_keys, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.pos, n, tb.sc, tb.key3, k0, tb.key2, i0,
                                                   multi ? tb.sys_id : nullptr, tb.sys_root, tb.single, 0);
        L += 1;
        cudaError_t e = sort_reset(tb.sort_scratch, n, st);
        if (e == cudaSuccess)
            e = sort_histograms(tb.key2, p2, 0, tb.key3, 8, 8, multi ? tb.sys_id : nullptr, 16, n, tb.sort_scratch,
                                nullptr, st, &L);
        if (e != cudaSuccess) return e;
        passes(k0, k0o, i0, i0o, p2, p2, 0, nullptr, st);                   // result: key_a, idx_a
        gather(tb.key3, tb.key_b, nullptr, st);                               // k1 in that order
        passes(tb.key_b, tb.key_a, tb.idx_a, tb.idx_b, 8, 8, 8, nullptr, st);  // result: key_b, idx_a
    } else {
        uint64_t *k0 = (p1 & 1) ? tb.key_a : tb.key_b, *k0o = (p1 & 1) ? tb.key_b : tb.key_a;
        uint32_t *i0 = (p1 & 1) ? tb.idx_b : tb.idx_a, *i0o = (p1 & 1) ? tb.idx_a : tb.idx_b;
        launch_pdl(k_keys, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.pos, n, tb.sc, tb.key3, k0, nullptr, i0, nullptr, tb.sys_root,
                                                   tb.single, 1);
        L += 1;
        cudaError_t e = sort_reset(tb.sort_scratch, n, st);
        if (e == cudaSuccess)
            e = sort_histograms(tb.key3, p1, 8, nullptr, 0, 0, nullptr, 0, n, tb.sort_scratch, nullptr, st, &L);
        if (e != cudaSuccess) return e;
        passes(k0, k0o, i0, i0o, p1, p1, 8, nullptr, st);  // result: key_b, idx_a
    }
    if (checked) {
        // Equal neighbours over the bits the plan sorted mean it did not separate
        // every particle: short runs of them are sorted in place, and a long one
        // makes the full sort run. Inside a stream capture the full sort is the
        // body of a conditional graph node that runs only when the check sets its
        // condition; launched directly, each of its kernels returns at once unless
        // the flag is set.
        if (p2 > 0) gather(tb.key2, tb.key_a, nullptr, st);  // k2 in sorted order, for the check and the runs
        cudaGraphConditionalHandle cond = 0;
        cudaGraph_t cg = nullptr;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const bool use_cond = tb.cond_stream && cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg) == cudaSuccess &&
                              cs == cudaStreamCaptureStatusActive &&
                              cudaGraphConditionalHandleCreate(&cond, cg, 0, cudaGraphCondAssignDefault) == cudaSuccess;
        if (!use_cond) cudaGetLastError();
        launch_pdl(k_fix_ties, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.key_b, tb.key_a, tb.idx_a, tb.pos,
                   p2 > 0 ? 1 : 0, p2 > 0 ? 0 : digit_shift(p1, 0), p2 > 0 ? digit_shift(p2, 0) : 0, n, tb.single,
                   tb.sc, cond, use_cond ? 1 : 0);
        L += 1;
        cudaStream_t fs = st;
        cudaError_t e;
        if (use_cond) {
            const cudaGraphNode_t *deps = nullptr;
            size_t ndeps = 0;
            if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps)) != cudaSuccess) return e;
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            if ((e = cudaGraphAddNode(&node, cg, deps, ndeps, &cp)) != cudaSuccess) return e;
            if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
                return e;
            if ((e = cudaStreamBeginCaptureToGraph(tb.cond_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed)) != cudaSuccess)
                return e;
            fs = tb.cond_stream;
        }
        // the full sort by (k1, k2): 8 passes on k2, the gather of k1, 8 passes on k1
        const unsigned body_first = L;
        if (p2 == 0) {
            launch_pdl(k_keys_second, dim3(blocks_for(n, 256)), dim3(256), 0, fs, tb.pos, n, tb.sc, tb.key2, tb.single, ties);
            L += 1;
        }
        if ((e = sort_histograms(tb.key2, 8, 18, tb.key3, 8, 26, nullptr, 0, n, tb.sort_scratch, ties, fs, &L)) !=
            cudaSuccess)
            return e;
        launch_pdl(k_full_sort_init, dim3(blocks_for(n, 256)), dim3(256), 0, fs, tb.key2, tb.key_a, tb.idx_a, n, ties);
        L += 1;
        passes(tb.key_a, tb.key_b, tb.idx_a, tb.idx_b, 8, 8, 18, ties, fs);  // result: key_a, idx_a
        gather(tb.key3, tb.key_b, ties, fs);
        passes(tb.key_b, tb.key_a, tb.idx_a, tb.idx_b, 8, 8, 26, ties, fs);  // result: key_b, idx_a
        gather(tb.key2, tb.key_a, ties, fs);                                  // k2 sorted
        if (use_cond) {
            cudaGraph_t body = nullptr;
            if ((e = cudaStreamEndCapture(fs, &body)) != cudaSuccess) return e;
            if (tb.cond_launches) *tb.cond_launches += L - body_first;
        }
    }
    if (multi) {
        // then by system (16-bit ids, 2 stable passes; result back in key_a / idx_a)
        launch_pdl(k_gather_sys, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.sys_id, tb.idx_a, tb.key_a, nullptr, n);
        passes(tb.key_a, tb.key_b, tb.idx_a, tb.idx_b, 2, 8, 16, nullptr, st);
        gather(tb.key3, tb.key_b, nullptr, st);  // k1 sorted
        launch_pdl(k_gather_sys, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.sys_id, tb.idx_a, nullptr, tb.sys_sorted, n);
        L += 2;
    }
    // k2 sorted into key_a (a checked plan has it already, or needs none: with
    // every k1 prefix distinct, nothing reads k2)
    if (!checked) gather(tb.key2, tb.key_a, nullptr, st);
    if (tb.mass_ready && !multi) cudaStreamWaitEvent(st, tb.mass_ready, 0);  // the first reader of the masses
    launch_pdl(k_gather_bodies, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.idx_a, tb.pos, tb.mass, tb.body, n, tb.sc, tb.single);
    L += 1;
    *launches += L;
    if (n < 2) return cudaGetLastError();
    L = 0;
    const uint32_t *sys_sorted = multi ? tb.sys_sorted : nullptr;
    launch_pdl(k_deep_groups, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.key_b, tb.key_a, tb.key3, tb.idx_a, tb.body, n,
                                                       sys_sorted, tb.sys_root, tb.sc, tb.single);
    KeyView kv{tb.key_b, tb.key_a, tb.key3, (int)n, sys_sorted};
    const uint32_t m = n - 1;
    launch_pdl(k_radix_tree, dim3(blocks_for(m, 256)), dim3(256), 0, st, kv, tb.bleft, tb.bright, tb.bparent, tb.leaf_bparent,
                                                      tb.bdelta, &tb.sc->max_prefix_bits, tb.sc->pair_passes);
    launch_pdl(k_head_flags, dim3(blocks_for(n, 256)), dim3(256), 0, st, tb.bparent, tb.bdelta, m, tb.head_flag,
               tb.head_id, tb.oparent, tb.leaf_oparent, tb.ocount);
    L += 3 + scan_exclusive(tb.head_id, m, tb.scan_tmp, &tb.sc->n_onodes, st);
    launch_pdl(k_collapse, dim3(blocks_for(m, 256)), dim3(256), 0, st, tb.bleft, tb.bright, tb.bdelta, tb.head_id, tb.head_flag,
                                                    m, tb.ochild, tb.ometa, tb.oparent, tb.leaf_oparent,
                                                    tb.sc);
    L += 1;
    if (multi) {
        launch_pdl(k_sys_roots, dim3(blocks_for(tb.nsys, 256)), dim3(256), 0, st, tb.sys_start, tb.head_flag, tb.head_id, tb.nsys,
                                                               tb.sys_root_node);
        L += 1;
    }
    *launches += L;
    return cudaGetLastError();
}

cudaError_t compute_com(const TreeBuild &tb, cudaStream_t st, unsigned *launches) {
    const uint32_t n = tb.n;
    if (n < 2) return cudaSuccess;
    // (the arrival counts were zeroed by the build's k_head_flags)
    if (tb.single)
        launch_pdl(k_com<float>, dim3(blocks_for(n - 1, 256)), dim3(256), 0, st, tb.body, tb.leaf_oparent, tb.oparent, tb.ochild,
                                                             tb.ometa, tb.onode, tb.ocount, n, tb.sc);
    else
        launch_pdl(k_com<double>, dim3(blocks_for(n - 1, 256)), dim3(256), 0, st, tb.body, tb.leaf_oparent, tb.oparent, tb.ochild,
                                                              tb.ometa, tb.onode, tb.ocount, n, tb.sc);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace nbody
