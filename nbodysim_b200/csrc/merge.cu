// Particle merging on the GPU: the reference's minimum node size pass
// (apply_minimum_size, src/main.cpp:1001-1060) and its collision capture and
// merge (src/main.cpp:386-396, 423-430, 475-516, 521-550).
//
// Both produce, per particle, a label: the user index of the particle that
// represents its merged group (itself when it is not merged). The merged
// values are stored at the representative, and a compaction keeps the
// representatives and the untouched particles in user order.
//
// Minimum size: the reference folds, bottom-up, every node whose side is below
// min_size into one particle (each node's children in child order,
// new = collide(new, child)). After the fold only the topmost such cells
// matter: a cell at the first level L* whose side is below min_size keeps one
// particle, the fold of its subtree. A chain node passes its one child's
// particle up unchanged, so the fold over the chain-free octree below the
// topmost branching node inside the cell is the reference's fold, bit for bit.
//
// Collisions: a particle records a pair with every leaf its walk accepts that
// lies closer than the collision range. A separate walk per particle replays
// the reference's FP64 opening test exactly, but only inside nodes that can
// hold a leaf within range (every particle of a node lies in its cube, within
// side * sqrt(3) of its centre of mass). Pairs become connected components
// (union-find, root = smallest user index). The reference merges the pairs in
// the iteration order of an unordered_set, so its result for a group of three
// or more depends on pointer hashes; here each component is folded in
// ascending user index. For a single pair the order does not matter
// (IEEE addition commutes), so the merged particle is the reference's bit for bit.
#include "merge.cuh"
#include "sort.cuh"
#include "tree.cuh"

namespace nbody {

namespace {

constexpr uint32_t kUnionRetries = 1u << 20;
constexpr int kFrames = kMaxLevels + 2;


struct Val {
    double x, y, z, vx, vy, vz, m;
};

// collide(a, b) (src/main.cpp:423-430) with weighted_average
// (src/vector.cpp:129-132): (a*ma + b*mb) / (ma + mb), mass ma + mb.
__device__ inline void collide_into(Val &a, const Val &b) {
    const double w = __dadd_rn(a.m, b.m);
    a.x = __ddiv_rn(__dadd_rn(__dmul_rn(a.x, a.m), __dmul_rn(b.x, b.m)), w);
    a.y = __ddiv_rn(__dadd_rn(__dmul_rn(a.y, a.m), __dmul_rn(b.y, b.m)), w);
    a.z = __ddiv_rn(__dadd_rn(__dmul_rn(a.z, a.m), __dmul_rn(b.z, b.m)), w);
    a.vx = __ddiv_rn(__dadd_rn(__dmul_rn(a.vx, a.m), __dmul_rn(b.vx, b.m)), w);
    a.vy = __ddiv_rn(__dadd_rn(__dmul_rn(a.vy, a.m), __dmul_rn(b.vy, b.m)), w);
    a.vz = __ddiv_rn(__dadd_rn(__dmul_rn(a.vz, a.m), __dmul_rn(b.vz, b.m)), w);
    a.m = w;
}

__device__ inline Val user_val(const double *pos, const double *vel, const double *mass, uint32_t u) {
    const size_t o = 3 * (size_t)u;
    return {pos[o], pos[o + 1], pos[o + 2], vel[o], vel[o + 1], vel[o + 2], mass[u]};
}

__device__ inline void store_merged(const MergeBufs &m, uint32_t r, const Val &v) {
    const size_t o = 3 * (size_t)r;
    m.mpos[o] = v.x; m.mpos[o + 1] = v.y; m.mpos[o + 2] = v.z;
    m.mvel[o] = v.vx; m.mvel[o + 1] = v.vy; m.mvel[o + 2] = v.vz;
    m.mmass[r] = v.m;
    m.rep[r] = 1u;
}

// distance() of src/vector.cpp:99-102 on (a - b), every operation rounded alone.
__device__ inline double exact_dist(double ax, double ay, double az, double bx, double by, double bz) {
    const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

__global__ void k_merge_init(MergeBufs m, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMcCount) m.counters[i] = 0u;
    if (i >= n) return;
    m.label[i] = i;
    m.rep[i] = 0u;
    m.flag[i] = 0u;
}

// One thread per octree node; the topmost nodes at or below level L* fold their subtree.
__global__ void k_min_size(Tree t, const int32_t *__restrict__ oparent, const double *__restrict__ vel,
                           double min_size, MergeBufs m) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (t.n < 2 || p >= t.sc->n_onodes) return;
    const double S = t.sc->root_side;
    int ls = 0;  // first level whose cells are smaller than min_size (sides halve exactly)
    while (ls <= kMaxLevels && !(S * exp2_neg(ls) < min_size)) ls++;
    if (meta_level(t.ometa[p]) < ls) return;
    if (p != 0) {
        const int32_t par = oparent[p];
        if (par < 0 || meta_level(t.ometa[par]) >= ls) return;
    }
    // post-order fold with an explicit stack of frames (levels strictly increase downwards)
    int node[kFrames], next[kFrames];
    bool has[kFrames];
    Val acc[kFrames];
    int top = 0;
    node[0] = (int)p; next[0] = 0; has[0] = false;
    uint32_t jmin = 0xffffffffu, jmax = 0, umin = 0xffffffffu;
    Val out{};
    bool done = false;
    for (uint32_t guard = 0; guard < 4 * t.n + 64 && !done; guard++) {
        const int q = node[top];
        if (next[top] >= meta_nchild(t.ometa[q])) {
            const Val v = acc[top];
            if (top == 0) {
                out = v;
                done = true;
                break;
            }
            top--;
            if (!has[top]) { acc[top] = v; has[top] = true; }
            else collide_into(acc[top], v);
            continue;
        }
        const int32_t ch = t.ochild[8 * q + next[top]++];
        if (ch < 0) {
            const uint32_t j = ~(uint32_t)ch;
            const double4 b = t.body[j];
            const uint32_t u = t.sidx[j];
            const size_t o = 3 * (size_t)u;
            const Val v{b.x, b.y, b.z, vel[o], vel[o + 1], vel[o + 2], b.w};
            jmin = min(jmin, j); jmax = max(jmax, j); umin = min(umin, u);
            if (!has[top]) { acc[top] = v; has[top] = true; }
            else collide_into(acc[top], v);
        } else if (top + 1 < kFrames) {
            top++;
            node[top] = ch; next[top] = 0; has[top] = false;
        } else {
            break;
        }
    }
    if (!done || umin == 0xffffffffu) {
        atomicOr(&m.counters[kMcStatus], kMergeStatusTree);
        return;
    }
    store_merged(m, umin, out);
    for (uint32_t j = jmin; j <= jmax; j++) m.label[t.sidx[j]] = umin;
    atomicAdd(&m.counters[kMcGroups], 1u);
}

// One thread per particle (Morton order): a stackless walk (parent links) that
// opens exactly what the reference opens, restricted to nodes that can hold a
// leaf within range.
__global__ void k_collide_find(Tree t, const int32_t *__restrict__ oparent, double theta, double range,
                               MergeBufs m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n || t.n < 2) return;
    const double4 bi = t.body[i];
    const double S = t.sc->root_side;
    int node = 0;
    bool enter = true;
    for (uint32_t guard = 0; guard < 4 * t.n + 16; guard++) {
        if (enter) {
            const double4 nd = t.onode[node];
            const int32_t meta = t.ometa[node];
            const double side = S * exp2_neg(meta_level(meta));
            const double d = exact_dist(nd.x, nd.y, nd.z, bi.x, bi.y, bi.z);
            bool open = !(d > (range + side * 1.7320508075688772) * (1.0 + 1e-9));
            if (open) open = __ddiv_rn(side, d) > theta;  // src/main.cpp:377
            if (open) {
                int first = -1;
                const int nch = meta_nchild(meta);
                for (int k = 0; k < nch; k++) {
                    const int32_t ch = t.ochild[8 * node + k];
                    if (ch >= 0) {
                        if (first < 0) first = ch;
                        continue;
                    }
                    const uint32_t j = ~(uint32_t)ch;
                    if (j == i) continue;  // a particle's own leaf is never accepted
                    const double4 bj = t.body[j];
                    if (exact_dist(bj.x, bj.y, bj.z, bi.x, bi.y, bi.z) < range) {  // src/main.cpp:386
                        const uint32_t ui = t.sidx[i], uj = t.sidx[j];
                        const uint32_t slot = atomicAdd(&m.counters[kMcPairs], 1u);
                        if (slot < m.pair_cap) m.pairs[slot] = make_uint2(min(ui, uj), max(ui, uj));
                    }
                }
                if (first >= 0) {
                    node = first;
                    continue;
                }
            }
        }
        // the next internal sibling, climbing while a node has none
        if (node == 0) return;
        const int32_t par = oparent[node];
        if (par < 0) break;
        const int nch = meta_nchild(t.ometa[par]);
        int k = 0;
        while (k < nch && t.ochild[8 * par + k] != node) k++;
        int nxt = -1;
        for (k++; k < nch; k++) {
            const int32_t ch = t.ochild[8 * par + k];
            if (ch >= 0) {
                nxt = ch;
                break;
            }
        }
        if (nxt >= 0) {
            node = nxt;
            enter = true;
        } else {
            node = par;
            enter = false;
        }
    }
    atomicOr(&m.counters[kMcStatus], kMergeStatusTree);
}

// Root of x. Links only ever point to a smaller index, so the chase ends
// within x steps; stale reads of concurrent links are still ancestors.
__device__ inline uint32_t uf_find(const uint32_t *label, uint32_t x) {
    for (;;) {
        const uint32_t y = *(const volatile uint32_t *)&label[x];
        if (y >= x) return x;
        x = y;
    }
}

__global__ void k_uf_union(MergeBufs m, uint32_t np) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const uint2 pr = m.pairs[k];
    m.flag[pr.x] = 1u;
    m.flag[pr.y] = 1u;
    for (uint32_t it = 0; it < kUnionRetries; it++) {
        const uint32_t ra = uf_find(m.label, pr.x), rb = uf_find(m.label, pr.y);
        if (ra == rb) return;
        const uint32_t lo = min(ra, rb), hi = max(ra, rb);
        if (atomicCAS(&m.label[hi], hi, lo) == hi) return;  // hi was still a root: linked
    }
    atomicOr(&m.counters[kMcStatus], kMergeStatusUnion);
}

// Flattens the endpoints' labels to their roots and copies the endpoint flags for the scan.
__global__ void k_uf_flatten(MergeBufs m, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t f = m.flag[i];
    if (f) m.label[i] = uf_find(m.label, i);
    m.offs[i] = f;
}

__global__ void k_endpoint_keys(MergeBufs m, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !m.flag[i]) return;
    const uint32_t k = m.offs[i];
    m.skey_a[k] = m.label[i];
    m.sidx_a[k] = i;
}

// One thread per component (segment of equal roots, ascending user index; the
// root is the smallest index, so it comes first).
__global__ void k_fold_components(MergeBufs m, uint32_t k, const double *__restrict__ pos,
                                  const double *__restrict__ vel, const double *__restrict__ mass) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= k) return;
    const uint64_t r = m.skey_a[q];
    if (q > 0 && m.skey_a[q - 1] == r) return;
    Val acc = user_val(pos, vel, mass, m.sidx_a[q]);
    for (uint32_t s = q + 1; s < k && m.skey_a[s] == r; s++) collide_into(acc, user_val(pos, vel, mass, m.sidx_a[s]));
    store_merged(m, (uint32_t)r, acc);
}

__global__ void k_keep_flags(MergeBufs m, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) m.offs[i] = m.label[i] == i ? 1u : 0u;
}

template <typename AccT>
__global__ void k_compact(MergeBufs m, uint32_t n, const double *__restrict__ pos, const double *__restrict__ vel,
                          const double *__restrict__ mass, const AccT *__restrict__ acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || m.label[i] != i) return;
    const uint32_t j = m.offs[i];
    AccT *acc2 = (AccT *)m.acc2;
    const size_t o = 3 * (size_t)i, p = 3 * (size_t)j;
    if (m.rep[i]) {  // a new particle: merged state, zero acceleration
        for (int c = 0; c < 3; c++) {
            m.pos2[p + c] = m.mpos[o + c];
            m.vel2[p + c] = m.mvel[o + c];
            acc2[p + c] = (AccT)0;
        }
        m.mass2[j] = m.mmass[i];
    } else {
        for (int c = 0; c < 3; c++) {
            m.pos2[p + c] = pos[o + c];
            m.vel2[p + c] = vel[o + c];
            acc2[p + c] = acc[o + c];
        }
        m.mass2[j] = mass[i];
    }
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t merge_begin(const MergeBufs &m, uint32_t n, cudaStream_t st, unsigned *launches) {
    k_merge_init<<<blocks_for(std::max<uint32_t>(n, kMcCount), 256), 256, 0, st>>>(m, n);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t merge_min_size(const MergeBufs &m, const Tree &t, const int32_t *oparent, const double *vel,
                           double min_size, cudaStream_t st, unsigned *launches) {
    if (t.n < 2) return cudaSuccess;
    k_min_size<<<blocks_for(t.n - 1, 128), 128, 0, st>>>(t, oparent, vel, min_size, m);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t collide_find(const MergeBufs &m, const Tree &t, const int32_t *oparent, double theta, double range,
                         cudaStream_t st, unsigned *launches) {
    if (t.n < 2) return cudaSuccess;
    k_collide_find<<<blocks_for(t.n, 128), 128, 0, st>>>(t, oparent, theta, range, m);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t collide_components(const MergeBufs &m, uint32_t n, uint32_t npairs, cudaStream_t st, unsigned *launches) {
    if (npairs == 0 || n == 0) return cudaSuccess;
    k_uf_union<<<blocks_for(npairs, 256), 256, 0, st>>>(m, npairs);
    k_uf_flatten<<<blocks_for(n, 256), 256, 0, st>>>(m, n);
    *launches += 2 + scan_exclusive(m.offs, n, m.scan_tmp, &m.counters[kMcInvolved], st);
    k_endpoint_keys<<<blocks_for(n, 256), 256, 0, st>>>(m, n);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t collide_fold(const MergeBufs &m, uint32_t k, const double *pos, const double *vel, const double *mass,
                         cudaStream_t st, unsigned *launches) {
    if (k == 0) return cudaSuccess;
    // stable LSD sort of the endpoints (ascending user index) by their 32-bit root
    cudaError_t e = sort_reset(m.sort_scratch, k, st);
    if (e == cudaSuccess)
        e = sort_histograms(m.skey_a, 8, 0, nullptr, 0, 0, nullptr, 0, k, m.sort_scratch, nullptr, st, launches);
    if (e != cudaSuccess) return e;
    uint64_t *kin = m.skey_a, *kout = m.skey_b;
    uint32_t *iin = m.sidx_a, *iout = m.sidx_b;
    for (int q = 0; q < 4; q++) {
        e = sort_pass(kin, iin, kout, iout, k, q, digit_shift(8, q), m.sort_scratch, &m.counters[kMcStatus], kMergeStatusSort,
                      nullptr, st, launches);
        if (e != cudaSuccess) return e;
        uint64_t *tk = kin; kin = kout; kout = tk;
        uint32_t *ti = iin; iin = iout; iout = ti;
    }
    // four passes: the result is back in skey_a / sidx_a
    k_fold_components<<<blocks_for(k, 256), 256, 0, st>>>(m, k, pos, vel, mass);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t merge_compact(const MergeBufs &m, uint32_t n, const double *pos, const double *vel, const double *mass,
                          const void *acc, bool acc_double, cudaStream_t st, unsigned *launches) {
    if (n == 0) return cudaSuccess;
    k_keep_flags<<<blocks_for(n, 256), 256, 0, st>>>(m, n);
    *launches += 1 + scan_exclusive(m.offs, n, m.scan_tmp, &m.counters[kMcKept], st);
    if (acc_double) k_compact<double><<<blocks_for(n, 256), 256, 0, st>>>(m, n, pos, vel, mass, (const double *)acc);
    else k_compact<float><<<blocks_for(n, 256), 256, 0, st>>>(m, n, pos, vel, mass, (const float *)acc);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace nbody
