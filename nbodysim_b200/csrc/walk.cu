// Fused Barnes-Hut walk + gravity, one warp per 32 Morton-consecutive particles.
//
// Semantics are the reference's per-particle BFS (src/main.cpp:368-400): a
// particle opens a node iff side / |com - x| > theta and the node is not a
// leaf, otherwise it accepts the node unless the node is its own leaf; an
// accepted node adds G M (com - x) / r^3 (src/main.cpp:306-333). Every lane
// keeps exactly its own decisions: the warp walks the union of the 32 walks,
// carrying with every stacked node the mask of lanes that reached it (opened
// all its ancestors). Lanes outside the mask ignore the node, so each lane's
// accepted set is the reference's set for that particle.
//
// The octree here has no single-child chains (tree.cu). A reference chain
// above a branching node K has K's mass and K's centre of mass (to rounding),
// and a larger side; a particle that opens K opens the whole chain, and one
// that does not accepts exactly one chain node -- the same body. So the
// accepted bodies and their count match the reference.
//
// MIXED precision: coordinates enter the inner loop as FP32 offsets from the
// group's bbox centre, pair forces and accumulation are FP32. The opening test
// r^2 < (side/theta)^2 is evaluated in FP32 with a proven error band; a lane
// whose value falls inside the band re-evaluates the reference's FP64
// expression exactly (side / sqrt(dx^2 + dy^2 + dz^2) > theta on the original
// doubles), so decisions are those of the FP64 reference.
// FP64 ("plain form"): the same walk with every quantity in FP64 and the
// reference's FP64 opening test evaluated directly.
#include "walk.cuh"

namespace nbody {

namespace {

constexpr float kU = 5.9604644775390625e-8f;  // 2^-24, FP32 unit roundoff
// Band half-width (see walk_band in the comments of k_walk): 32u q + 20u Pm sqrt(q),
// plus every r^2 below (64 u Pm)^2.
constexpr float kTolRel = 32.0f * kU;
constexpr float kTolPm = 20.0f * kU;
constexpr float kTiny = 64.0f * kU;

__device__ inline double exp2_neg(int L) {  // exactly 2^-L for 0 <= L <= 1022
    return __longlong_as_double((long long)(1023 - L) << 52);
}

template <bool kFp64>
struct WarpTiles;

template <>
struct WarpTiles<false> {
    int2 stack[kStackCap];
    float4 c[32];      // (com - ref).xyz, G m
    float4 q[32];      // q = (side/theta)^2, sqrt(q), 32u q, -
    int2 r[32];        // node ref, reach mask
    int child[32][8];  // children of internal entries
    int nch[32];
};

template <>
struct WarpTiles<true> {
    int2 stack[kStackCap];
    double4 c[32];     // com.xyz (absolute), G m
    double side[32];   // node side (internal), -1 for leaves
    int2 r[32];
    int child[32][8];
    int nch[32];
};

// The reference's FP64 opening test on the original doubles
// (src/main.cpp:377 with distance() of src/vector.cpp:99-102).
__device__ inline bool exact_open(double cx, double cy, double cz, double px, double py, double pz,
                                  double side, double theta) {
    double dx = __dsub_rn(cx, px), dy = __dsub_rn(cy, py), dz = __dsub_rn(cz, pz);
    double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    return __ddiv_rn(side, d) > theta;
}

// Moves the oldest half of a full stack to this warp's global spill region.
template <class Tiles>
__device__ inline bool spill_out(Tiles &s, int &top, uint32_t &spill_top, int2 *gspill,
                                 uint32_t spill_cap, int lane) {
    if (spill_top + kSpillChunk > spill_cap) return false;
    for (int e = lane; e < kSpillChunk; e += 32) gspill[spill_top + e] = s.stack[e];
    __syncwarp();
    for (int e = lane; e < top - kSpillChunk; e += 32) s.stack[e] = s.stack[e + kSpillChunk];
    __syncwarp();
    top -= kSpillChunk;
    spill_top += kSpillChunk;
    return true;
}

template <class Tiles>
__device__ inline void spill_in(Tiles &s, int &top, uint32_t &spill_top, const int2 *gspill, int lane) {
    int take = min((int)spill_top, kSpillChunk);
    for (int e = lane; e < take; e += 32) s.stack[e] = gspill[spill_top - take + e];
    __syncwarp();
    spill_top -= take;
    top = take;
}

template <bool kFp64, bool kDamp, bool kPot>
__global__ void __launch_bounds__(kWalkWarps * 32) k_walk(WalkArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using Tiles = WarpTiles<kFp64>;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    Tiles &s = reinterpret_cast<Tiles *>(smem_raw)[wid];
    const Tree &t = a.t;
    const uint32_t n = t.n;
    const double S = t.sc->root_side;
    const double theta = a.theta;
    const double s_theta = S / theta;
    int2 *gspill = a.spill + (size_t)(blockIdx.x * kWalkWarps + wid) * a.spill_cap;
    const unsigned FULL = 0xffffffffu;

    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(&t.sc->group_counter, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= a.n_groups) break;

        const uint32_t j = g * 32 + lane;
        const bool valid = j < n;
        const double4 b = t.body[valid ? j : g * 32];
        const uint32_t vmask = __ballot_sync(FULL, valid);

        // Reference point: centre of the group's bounding box.
        const double rx = 0.5 * (warp_min(b.x) + warp_max(b.x));
        const double ry = 0.5 * (warp_min(b.y) + warp_max(b.y));
        const double rz = 0.5 * (warp_min(b.z) + warp_max(b.z));
        const float px = (float)(b.x - rx), py = (float)(b.y - ry), pz = (float)(b.z - rz);
        // Error band of the FP32 test (walk_band): with u = 2^-24 and Pm the
        // largest |offset| of this particle, |r2_f32 - r2| <= 7.1u r2 + 7u Pm sqrt(r2)
        // and |q_f32 - q| <= 1.01u q, so outside |r2 - q| <= 32u q + 20u Pm sqrt(q)
        // and r2 > (64u Pm)^2 the FP32 decision equals the exact one.
        const float pm = fmaxf(fabsf(px), fmaxf(fabsf(py), fabsf(pz)));
        const float pm_tol = kTolPm * pm;
        const float tiny = (kTiny * pm) * (kTiny * pm);

        float fax = 0.f, fay = 0.f, faz = 0.f, fpot = 0.f;
        double dax = 0.0, day = 0.0, daz = 0.0, dpot = 0.0;
        uint32_t cnt = 0, nfallback = 0;
        int top = 0;
        uint32_t spill_top = 0;
        int max_top = 0;
        bool failed = false;
        if (n >= 2) {
            if (lane == 0) s.stack[0] = make_int2(0, (int)vmask);
            top = 1;
        }
        __syncwarp();

        while (top > 0 || spill_top > 0) {
            if (top == 0) spill_in(s, top, spill_top, gspill, lane);
            const int cntt = min(top, 32);
            const int base = top - cntt;
            top = base;
            // ---- stage a tile of up to 32 stacked nodes in shared memory
            if (lane < cntt) {
                const int2 e = s.stack[base + lane];
                double cx, cy, cz, m;
                int nch = 0;
                double so = -1.0;
                if (e.x >= 0) {
                    const double4 nd = t.onode[e.x];
                    const int meta = t.ometa[e.x];
                    cx = nd.x; cy = nd.y; cz = nd.z; m = nd.w;
                    nch = meta_nchild(meta);
                    const double sc2 = exp2_neg(meta_level(meta));
                    so = kFp64 ? S * sc2 : s_theta * sc2;
                    const int4 *cp = reinterpret_cast<const int4 *>(t.ochild + 8 * (size_t)e.x);
                    const int4 c0 = cp[0], c1 = cp[1];
                    s.child[lane][0] = c0.x; s.child[lane][1] = c0.y;
                    s.child[lane][2] = c0.z; s.child[lane][3] = c0.w;
                    s.child[lane][4] = c1.x; s.child[lane][5] = c1.y;
                    s.child[lane][6] = c1.z; s.child[lane][7] = c1.w;
                } else {
                    const double4 bd = t.body[~e.x];
                    cx = bd.x; cy = bd.y; cz = bd.z; m = bd.w;
                }
                if constexpr (kFp64) {
                    s.c[lane] = make_double4(cx, cy, cz, kG * m);
                    s.side[lane] = so;  // node side, or -1 for a leaf
                } else {
                    s.c[lane] = make_float4((float)(cx - rx), (float)(cy - ry), (float)(cz - rz),
                                            (float)(kG * m));
                    if (so > 0.0) {
                        const float qf = (float)(so * so);
                        s.q[lane] = make_float4(qf, (float)so, kTolRel * qf, 0.f);
                    } else {
                        s.q[lane] = make_float4(-1.f, 0.f, 0.f, 0.f);
                    }
                }
                s.r[lane] = e;
                s.nch[lane] = nch;
            }
            __syncwarp();
            // ---- every lane tests every node of the tile against its particle
            for (int k = 0; k < cntt; k++) {
                const int2 rm = s.r[k];
                const bool reached = (rm.y >> lane) & 1;
                bool open = false;
                bool take;
                if constexpr (kFp64) {
                    const double4 c = s.c[k];
                    const double dx = __dsub_rn(c.x, b.x), dy = __dsub_rn(c.y, b.y),
                                 dz = __dsub_rn(c.z, b.z);
                    const double r2 =
                        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    double d = -1.0;
                    if (rm.x >= 0) {
                        d = __dsqrt_rn(r2);
                        open = __ddiv_rn(s.side[k], d) > theta;
                    }
                    take = reached && !open && rm.x != (int)~j;
                    if (__any_sync(FULL, take) && take) {
                        if (d < 0.0) d = sqrt(r2);
                        const double inv = 1.0 / d;
                        double f;
                        if constexpr (kDamp) f = c.w * inv / (r2 + exp(-d));
                        else f = c.w * inv * inv * inv;
                        dax = fma(f, dx, dax); day = fma(f, dy, day); daz = fma(f, dz, daz);
                        if constexpr (kPot) dpot += c.w * inv;
                        cnt++;
                    }
                } else {
                    const float4 c = s.c[k];
                    const float dx = c.x - px, dy = c.y - py, dz = c.z - pz;
                    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    if (rm.x >= 0) {
                        const float4 q = s.q[k];
                        const float dq = r2 - q.x;
                        open = dq < 0.f;
                        const bool amb = reached && (fabsf(dq) <= fmaf(pm_tol, q.y, q.z) || r2 <= tiny);
                        if (__any_sync(FULL, amb) && amb) {
                            const double4 nd = t.onode[rm.x];
                            const double side = S * exp2_neg(meta_level(t.ometa[rm.x]));
                            open = exact_open(nd.x, nd.y, nd.z, b.x, b.y, b.z, side, theta);
                            nfallback++;
                        }
                    }
                    take = reached && !open && rm.x != (int)~j;
                    if (__any_sync(FULL, take) && take) {
                        const float inv = rsqrtf(r2);
                        float f;
                        if constexpr (kDamp) {
                            const float r = r2 * inv;
                            f = c.w * inv / (r2 + expf(-r));
                        } else {
                            f = c.w * inv * inv * inv;
                        }
                        fax = fmaf(f, dx, fax); fay = fmaf(f, dy, fay); faz = fmaf(f, dz, faz);
                        if constexpr (kPot) fpot = fmaf(c.w, inv, fpot);
                        cnt++;
                    }
                }
                const uint32_t openm = __ballot_sync(FULL, reached && open);
                if (openm) {
                    const int nch = s.nch[k];
                    if (top + nch > kStackCap) {
                        if (!spill_out(s, top, spill_top, gspill, a.spill_cap, lane)) {
                            failed = true;
                            break;
                        }
                    }
                    if (lane < nch) s.stack[top + lane] = make_int2(s.child[k][lane], (int)openm);
                    top += nch;
                    max_top = max(max_top, top + (int)spill_top);
                    __syncwarp();
                }
            }
            __syncwarp();
            if (failed) break;
        }
        if (failed && lane == 0) atomicOr(&t.sc->status, kStatusCapacity);

        // ---- epilogue: results in the caller's particle order
        double ax, ay, az;
        if constexpr (kFp64) { ax = dax; ay = day; az = daz; }
        else { ax = fax; ay = fay; az = faz; }
        if (valid) {
            const uint32_t ui = t.sidx[j];
            if constexpr (kFp64) {
                a.accd[3 * (size_t)ui] = ax; a.accd[3 * (size_t)ui + 1] = ay; a.accd[3 * (size_t)ui + 2] = az;
            } else {
                a.accf[3 * (size_t)ui] = fax; a.accf[3 * (size_t)ui + 1] = fay; a.accf[3 * (size_t)ui + 2] = faz;
            }
            if (a.counts) a.counts[ui] = cnt;
            if constexpr (kPot) {
                if (a.pot) a.pot[ui] = kFp64 ? -dpot : -(double)fpot;
            }
        }
        unsigned long long wc = cnt;
        for (int o = 16; o; o >>= 1) wc += __shfl_xor_sync(FULL, wc, o);
        uint32_t wf = nfallback;
        for (int o = 16; o; o >>= 1) wf += __shfl_xor_sync(FULL, wf, o);
        double amag = valid ? sqrt(ax * ax + ay * ay + az * az) : 0.0;
        if (a.track_max_acc) amag = warp_max(amag);
        if (lane == 0) {
            atomicAdd(&t.sc->interactions, wc);
            atomicAdd(&t.sc->interactions_total, wc);
            if (wf) atomicAdd(&t.sc->fallback_tests, wf);
            atomicMax(&t.sc->max_stack, (uint32_t)max_top);
            if (a.track_max_acc) atomic_max_nonneg(&t.sc->max_acc_bits, amag);
        }
        (void)vmask;
    }
}

template <bool kFp64>
const void *walk_kernel(int damping, bool pot) {
    if (damping) return pot ? (const void *)k_walk<kFp64, true, true> : (const void *)k_walk<kFp64, true, false>;
    return pot ? (const void *)k_walk<kFp64, false, true> : (const void *)k_walk<kFp64, false, false>;
}

}  // namespace

cudaError_t walk_launch_shape(bool fp64, int device, WalkLaunch *out) {
    const size_t smem = (fp64 ? sizeof(WarpTiles<true>) : sizeof(WarpTiles<false>)) * kWalkWarps;
    const void *kernels[8] = {
        (const void *)k_walk<false, false, false>, (const void *)k_walk<false, false, true>,
        (const void *)k_walk<false, true, false>, (const void *)k_walk<false, true, true>,
        (const void *)k_walk<true, false, false>, (const void *)k_walk<true, false, true>,
        (const void *)k_walk<true, true, false>, (const void *)k_walk<true, true, true>};
    int minblocks = 1 << 30;
    for (int k = 0; k < 8; k++) {
        cudaError_t e = cudaFuncSetAttribute(kernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    for (int k = fp64 ? 4 : 0; k < (fp64 ? 8 : 4); k++) {
        int nb = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernels[k], kWalkWarps * 32, smem);
        if (e != cudaSuccess) return e;
        minblocks = nb < minblocks ? nb : minblocks;
    }
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    if (minblocks < 1) minblocks = 1;
    out->blocks = (unsigned)(sms * minblocks);
    out->smem = smem;
    return cudaSuccess;
}

cudaError_t launch_walk(const WalkArgs &a, bool fp64, const WalkLaunch &l, cudaStream_t st) {
    const void *k = fp64 ? walk_kernel<true>(a.damping, a.pot != nullptr)
                         : walk_kernel<false>(a.damping, a.pot != nullptr);
    unsigned blocks = l.blocks;
    const unsigned need = (a.n_groups + kWalkWarps - 1) / kWalkWarps;
    if (need < blocks) blocks = need ? need : 1;
    WalkArgs args = a;
    void *params[] = {&args};
    return cudaLaunchKernel(k, dim3(blocks), dim3(kWalkWarps * 32), params, l.smem, st);
}

}  // namespace nbody
