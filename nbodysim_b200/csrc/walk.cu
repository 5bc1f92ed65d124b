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
// whose value falls inside the band re-evaluates the reference's expression
// exactly (side / sqrt(dx^2 + dy^2 + dz^2) > theta on the original values, in
// the arithmetic of the reference build: FP64, or the FLOAT build's float), so
// decisions are those of the reference.
// Accepted bodies go to one of three lists, each stored as pairs of entries
// for the packed FP32 instructions (two entries per instruction): entries that
// every lane of the group takes (no mask), entries some lanes take (a lane mask
// each), and bodies close to the group's box, whose offsets carry an FP32
// remainder so that close pairs keep FP32 accuracy of the offset itself.
// FP64 ("plain form"): the same walk with every quantity in FP64 and the
// reference's opening test evaluated directly.
#include "walk.cuh"

namespace nbody {

namespace {

constexpr float kU = 5.9604644775390625e-8f;  // 2^-24, FP32 unit roundoff
// Band half-width (see walk_band in the comments of k_walk): 32u q + 20u Pm sqrt(q),
// plus every r^2 below (64 u Pm)^2.
constexpr float kTolRel = 32.0f * kU;
constexpr float kTolPm = 20.0f * kU;
constexpr float kTiny = 64.0f * kU;

// 1/sqrt(x) in one special-function instruction (flush-to-zero; squared pair
// distances are never subnormal), the same ~2 ulp accuracy as rsqrtf without
// rsqrtf's subnormal fix-up instructions.
__device__ inline float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}


// Per-warp shared memory. The stack holds nodes still to be examined with
// the mask of lanes that reached them; the tile holds the up-to-32 internal
// nodes being decided; the list holds accepted bodies (internal nodes a lane
// did not open, and leaves) with the mask of lanes that take them.
template <bool kFp64>
struct WarpSmem;

// Values that are the same for every lane of a group, kept in shared memory
// rather than in one register per lane.
struct GroupConsts {
    double ref[3];      // reference point: centre of the group's bounding box
    double S, s_theta;  // root side, root side / theta
    float box[6];       // group box of the FP32 offsets: lo x, hi x, lo y, hi y, lo z, hi z
    float pm_tol, tiny, near_r2, pad;
    uint32_t st[6];     // per-group statistics: entries, tiles, decisions, list, near, deepest stack
};

// MIXED lists of the forward walk are stored in pairs of entries, so that the
// packed FP32 instructions (two lanes of arithmetic each) read their operands
// straight from two 16-byte loads: entries 2j and 2j+1 occupy 8 floats
// (x0, x1, y0, y1, z0, z1, Gm0, Gm1) at 8j. The adjoint keeps one float4 per entry.
template <>
struct WarpSmem<false> {
    GroupConsts gc;
    int2 stack[kStackCap];
    // The tile's mixed nodes, compacted and stored in pairs: pair j holds
    // x0 x1 y0 y1 z0 z1 -q0 -q1 band0 band1 reach0 reach1 ref0 ref1 - - at 16 j
    // ((com - ref).xyz, q = (side/theta)^2, the half-width of its error band, the
    // mask of lanes that reached the node, the node). Once a pair is decided,
    // its first two words hold the two open masks.
    alignas(16) float mx[16 * 16];
    union {
        float4 lc[kListCap];  // adjoint: (com - ref).xyz, G m per entry
        float lp[4 * kListCap];  // forward: entries taken by some lanes, in pairs
    };
    float lf[4 * kListCap];   // forward: entries taken by every lane of the group, in pairs
    uint32_t lm[kListCap];
    int lr[kListCap];         // node refs (adjoint mode)
    union {
        double4 nc[32];       // adjoint near list: com.xyz (absolute), G m
        struct {
            float hi[4 * kListCap];  // forward near list, in pairs: offsets rounded to FP32, G m
            float lo[4 * kListCap];  // and what the rounding left (x, y, z; the fourth slot is 0)
        } np;
    };
    uint32_t nm[kListCap];
    int nr[32];
};

// The paired lists and the mixed-node pairs are read with 16-byte loads.
static_assert(offsetof(WarpSmem<false>, mx) % 16 == 0 && offsetof(WarpSmem<false>, lp) % 16 == 0 &&
                  offsetof(WarpSmem<false>, lf) % 16 == 0 && offsetof(WarpSmem<false>, np) % 16 == 0 &&
                  sizeof(WarpSmem<false>) % 16 == 0,
              "16-byte shared loads need 16-byte aligned arrays");

template <>
struct WarpSmem<true> {
    GroupConsts gc;
    int2 stack[kStackCap];
    double4 tc[32];           // com.xyz (absolute), side
    int2 tr[32];              // reach mask, node ref
    double4 lc[kListCap];     // com.xyz (absolute), G m
    uint32_t lm[kListCap];
    int lr[kListCap];
};

// The reference's FP64 opening test on the original doubles
// (src/main.cpp:377 with distance() of src/vector.cpp:99-102).
__device__ inline bool exact_open(double cx, double cy, double cz, double px, double py, double pz,
                                  double side, double theta) {
    double dx = __dsub_rn(cx, px), dy = __dsub_rn(cy, py), dz = __dsub_rn(cz, pz);
    double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    return __ddiv_rn(side, d) > theta;
}

// The same test as the reference's FLOAT build evaluates it: float
// differences, their squares summed in double (pow(float, 2) promotes), the
// double square root rounded to float, then float side / float distance
// against float theta (src/main.cpp:377, src/vector.cpp:99-102, datatype float).
__device__ inline bool exact_open_f32(double cx, double cy, double cz, double px, double py, double pz,
                                      double side, float theta) {
    const float dx = __fsub_rn((float)cx, (float)px), dy = __fsub_rn((float)cy, (float)py),
                dz = __fsub_rn((float)cz, (float)pz);
    const double s = __dadd_rn(__dadd_rn(__dmul_rn((double)dx, (double)dx), __dmul_rn((double)dy, (double)dy)),
                               __dmul_rn((double)dz, (double)dz));
    const float d = __double2float_rn(__dsqrt_rn(s));
    return __fdiv_rn(__double2float_rn(side), d) > theta;
}

// The reference's opening test in the build's datatype.
__device__ inline bool ref_open(bool single, double cx, double cy, double cz, double px, double py, double pz,
                                double side, double theta, float theta_f) {
    return single ? exact_open_f32(cx, cy, cz, px, py, pz, side, theta_f)
                  : exact_open(cx, cy, cz, px, py, pz, side, theta);
}

// Moves the oldest half of a full stack to this warp's global spill region.
template <class Sm>
__device__ inline bool spill_out(Sm &s, int &top, uint32_t &spill_top, int2 *gspill, uint32_t spill_cap,
                                 int lane) {
    if (spill_top + kSpillChunk > spill_cap) return false;
    for (int e = lane; e < kSpillChunk; e += 32) gspill[spill_top + e] = s.stack[e];
    __syncwarp();
    for (int e = lane; e < top - kSpillChunk; e += 32) s.stack[e] = s.stack[e + kSpillChunk];
    __syncwarp();
    top -= kSpillChunk;
    spill_top += kSpillChunk;
    return true;
}

template <class Sm>
__device__ inline void spill_in(Sm &s, int &top, uint32_t &spill_top, const int2 *gspill, int lane) {
    int take = min((int)spill_top, kSpillChunk);
    for (int e = lane; e < take; e += 32) s.stack[e] = gspill[spill_top - take + e];
    __syncwarp();
    spill_top -= take;
    top = take;
}

// ---- packed FP32 pairs (sm_100 f32x2: one instruction, two FP32 lanes of work)
__device__ inline uint64_t f2pack(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ inline void f2unpack(uint64_t r, float &a, float &b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
__device__ inline uint64_t f2add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ inline uint64_t f2mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ inline uint64_t f2fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Writes entry k of a paired list.
__device__ inline void put_pair_entry(float *l, int k, float x, float y, float z, float gm) {
    float *e = l + 8 * (k >> 1) + (k & 1);
    e[0] = x; e[2] = y; e[4] = z; e[6] = gm;
}

// An offset o (FP64) as hi + lo in FP32: hi = o rounded, lo = what it left, rounded.
__device__ inline float lo_part(double o, float hi) { return (float)(o - (double)hi); }

// Gravity of the entries of a paired list on this lane's particle, two entries
// per packed instruction. kMasked: entry k is taken iff `bit` is set in lm[k];
// an entry not taken enters with inverse distance 0, so it adds exactly 0 even
// when it is the lane's own leaf (distance 0). Without kMasked every entry is
// taken. An odd count is padded with a far, massless entry. Accumulates into
// (ax, ay, az).
//
// kComp (the near list): the entry offsets are hi + lo pairs (`lo` holds the lo
// parts in the same layout) and so is the particle's (plx, ply, plz): the
// difference is (hi - phi) + (lo - plo). When hi and phi are within a factor
// two of each other their difference is exact (Sterbenz), so a body close to
// the particle gets its offset to FP32 accuracy of the offset itself.
template <bool kDamp, bool kMasked, bool kComp = false>
__device__ inline void force_pairs_f32(float *l, const uint32_t *lm, int count, uint32_t bit, float px, float py,
                                       float pz, float &ax, float &ay, float &az, float *lo = nullptr,
                                       float plx = 0.f, float ply = 0.f, float plz = 0.f) {
    if (count & 1) {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            put_pair_entry(l, count, 1e18f, 1e18f, 1e18f, 0.f);
            if constexpr (kComp) put_pair_entry(lo, count, 0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
    }
    const uint64_t npx = f2pack(-px, -px), npy = f2pack(-py, -py), npz = f2pack(-pz, -pz);
    uint64_t nlx = 0, nly = 0, nlz = 0;
    if constexpr (kComp) { nlx = f2pack(-plx, -plx); nly = f2pack(-ply, -ply); nlz = f2pack(-plz, -plz); }
    uint64_t sx = f2pack(0.f, 0.f), sy = sx, sz = sx;
    const int pairs = (count + 1) >> 1;
#pragma unroll 2
    for (int j = 0; j < pairs; j++) {
        const float4 A = *reinterpret_cast<const float4 *>(l + 8 * j);      // x0 x1 y0 y1
        const float4 B = *reinterpret_cast<const float4 *>(l + 8 * j + 4);  // z0 z1 g0 g1
        const float g0 = B.z, g1 = B.w;
        uint64_t dx = f2add(f2pack(A.x, A.y), npx);
        uint64_t dy = f2add(f2pack(A.z, A.w), npy);
        uint64_t dz = f2add(f2pack(B.x, B.y), npz);
        if constexpr (kComp) {
            const float4 C = *reinterpret_cast<const float4 *>(lo + 8 * j);
            const float4 D = *reinterpret_cast<const float4 *>(lo + 8 * j + 4);
            dx = f2add(dx, f2add(f2pack(C.x, C.y), nlx));
            dy = f2add(dy, f2add(f2pack(C.z, C.w), nly));
            dz = f2add(dz, f2add(f2pack(D.x, D.y), nlz));
        }
        const uint64_t r2 = f2fma(dz, dz, f2fma(dy, dy, f2mul(dx, dx)));
        float r0, r1;
        f2unpack(r2, r0, r1);
        float i0 = rsqrt_ftz(r0), i1 = rsqrt_ftz(r1);
        if constexpr (kMasked) {
            const uint2 m = *reinterpret_cast<const uint2 *>(lm + 2 * j);
            i0 = (m.x & bit) ? i0 : 0.f;
            i1 = (m.y & bit) ? i1 : 0.f;
        }
        uint64_t f;
        if constexpr (kDamp) {
            const float q0 = r0 * i0, q1 = r1 * i1;
            f = f2pack(g0 * i0 / (r0 + expf(-q0)), g1 * i1 / (r1 + expf(-q1)));
        } else {
            const uint64_t inv = f2pack(i0, i1);
            f = f2mul(f2mul(f2mul(inv, inv), inv), f2pack(g0, g1));
        }
        sx = f2fma(f, dx, sx);
        sy = f2fma(f, dy, sy);
        sz = f2fma(f, dz, sz);
    }
    float a0, a1;
    f2unpack(sx, a0, a1); ax += a0 + a1;
    f2unpack(sy, a0, a1); ay += a0 + a1;
    f2unpack(sz, a0, a1); az += a0 + a1;
}

// Per-particle accepted-body counts of a list (only when counts are requested).
__device__ inline uint32_t count_list(const uint32_t *lm, int count, uint32_t bit) {
    uint32_t c = 0;
    for (int k = 0; k < count; k++) c += (lm[k] & bit) ? 1u : 0u;
    return c;
}

// ---- adjoint pair terms (frozen decisions) --------------------------------
// For a taken pair with offset d = com - x and cotangent la = dL/da_i:
//   F = G M g(r) d,  dF/dd = G M (g I + h d d^T),  h = g'(r) / r,  dF/dM = G g d
//   undamped g = r^-3, h = -3 r^-5; damped g = 1 / (r (r^2 + e^-r)).
// v = (dF/dd) la goes to the node's centre-of-mass cotangent and, negated, to
// the particle's own position; G g (d . la) goes to the node's mass cotangent.
template <bool kDamp, typename T>
__device__ inline void pair_adjoint(T dx, T dy, T dz, T r2, T gm, T lax, T lay, T laz, T &vx, T &vy, T &vz,
                                    T &mterm) {
    if constexpr (sizeof(T) == 4) {
        // FP32: the same terms written with the unit offset u = d / r, so that no
        // factor grows faster than the force itself (h alone, ~ r^-5, overflows
        // FP32 below r ~ 2e-8): h s d = (h r^2) (u . la) u, G g s = G (g r) (u . la).
        const float inv = rsqrt_ftz(r2);
        const float ux = dx * inv, uy = dy * inv, uz = dz * inv;
        const float sh = ux * lax + uy * lay + uz * laz;
        float g, gr, hr2;
        if constexpr (kDamp) {
            const float r = r2 * inv;
            const float e = expf(-r);
            const float den = r2 + e;
            g = inv / den;
            gr = 1.f / den;
            hr2 = -(3.f * r2 + e - r * e) * inv / (den * den);
        } else {
            gr = inv * inv;
            g = gr * inv;
            hr2 = -3.f * g;
        }
        const float c = hr2 * sh;
        vx = gm * (g * lax + c * ux);
        vy = gm * (g * lay + c * uy);
        vz = gm * (g * laz + c * uz);
        mterm = float(kG) * gr * sh;
    } else {
        const T inv = 1.0 / sqrt(r2);
        const T inv2 = inv * inv;
        T g, h;
        if constexpr (kDamp) {
            const T r = r2 * inv;
            const T e = exp(-r);
            const T den = r2 + e;
            g = inv / den;
            h = -(T(3) * r2 + e - r * e) * inv2 * inv / (den * den);
        } else {
            g = inv * inv2;
            h = T(-3) * g * inv2;
        }
        const T s = dx * lax + dy * lay + dz * laz;
        const T hs = h * s;
        vx = gm * (g * lax + hs * dx);
        vy = gm * (g * lay + hs * dy);
        vz = gm * (g * laz + hs * dz);
        mterm = T(kG) * g * s;
    }
}

// Sums 32 per-lane values over the warp: lane l returns the sum over lanes of
// v[l]. Five butterfly stages (16 + 8 + 4 + 2 + 1 shuffles); at each stage a
// lane keeps the half of its values whose index has its own lane bit and sends
// the other half to its partner, so the 32 sums come out one per lane with
// only five dependent shuffles.
template <typename T>
__device__ inline T warp_transpose_sum32(T (&v)[32], int lane) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool h = lane & o;
#pragma unroll
        for (int i = 0; i < o; i++) {
            const T send = h ? v[i] : v[i + o];
            const T keep = h ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

// Lane l holds the warp sum of component (l & 3) of entry (l >> 2) of a chunk of
// eight: adds it to that node's (or leaf's) cotangent (x, y, z, mass).
__device__ inline void scatter_adj8(double *adj_node, double *adj_leaf, const int *lr, int k0, int count, double z,
                                    int lane) {
    const int k = k0 + (lane >> 2);
    if (k < count) {
        const int ref = lr[k];
        double *dst = ref >= 0 ? adj_node + 4 * (size_t)ref : adj_leaf + 4 * (size_t)(~ref);
        atomicAdd(dst + (lane & 3), z);
    }
}

// The list in chunks of eight entries: every lane's pair terms for the chunk,
// one transposed warp reduction, one atomic per lane.
template <bool kDamp>
__device__ inline void adj_list_f32(const float4 *lc, const uint32_t *lm, const int *lr, int count, int lane,
                                    float px, float py, float pz, float lax, float lay, float laz, float &gx,
                                    float &gy, float &gz, double *adj_node, double *adj_leaf) {
    for (int k0 = 0; k0 < count; k0 += 8) {
        float v[32];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int k = k0 + j;
            float vx = 0.f, vy = 0.f, vz = 0.f, mt = 0.f;
            if (k < count) {
                const float4 c = lc[k];
                const bool take = (lm[k] >> lane) & 1u;
                const float dx = c.x - px, dy = c.y - py, dz = c.z - pz;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                pair_adjoint<kDamp, float>(dx, dy, dz, r2, c.w, lax, lay, laz, vx, vy, vz, mt);
                if (!take) vx = vy = vz = mt = 0.f;
            }
            gx -= vx; gy -= vy; gz -= vz;
            v[4 * j] = vx; v[4 * j + 1] = vy; v[4 * j + 2] = vz; v[4 * j + 3] = mt;
        }
        const float z = warp_transpose_sum32(v, lane);
        scatter_adj8(adj_node, adj_leaf, lr, k0, count, (double)z, lane);
    }
}

template <bool kDamp>
__device__ inline void adj_near_f32(const double4 *nc, const uint32_t *nm, const int *nr, int count, int lane,
                                    double bx, double by, double bz, float lax, float lay, float laz, float &gx,
                                    float &gy, float &gz, double *adj_node, double *adj_leaf) {
    for (int k0 = 0; k0 < count; k0 += 8) {
        float v[32];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int k = k0 + j;
            float vx = 0.f, vy = 0.f, vz = 0.f, mt = 0.f;
            if (k < count && ((nm[k] >> lane) & 1u)) {
                const double4 c = nc[k];
                const float dx = (float)(c.x - bx), dy = (float)(c.y - by), dz = (float)(c.z - bz);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                pair_adjoint<kDamp, float>(dx, dy, dz, r2, (float)c.w, lax, lay, laz, vx, vy, vz, mt);
            }
            gx -= vx; gy -= vy; gz -= vz;
            v[4 * j] = vx; v[4 * j + 1] = vy; v[4 * j + 2] = vz; v[4 * j + 3] = mt;
        }
        const float z = warp_transpose_sum32(v, lane);
        scatter_adj8(adj_node, adj_leaf, nr, k0, count, (double)z, lane);
    }
}

template <bool kDamp>
__device__ inline void adj_list_f64(const double4 *lc, const uint32_t *lm, const int *lr, int count, int lane,
                                    double bx, double by, double bz, double lax, double lay, double laz, double &gx,
                                    double &gy, double &gz, double *adj_node, double *adj_leaf) {
    for (int k0 = 0; k0 < count; k0 += 8) {
        double v[32];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int k = k0 + j;
            double vx = 0.0, vy = 0.0, vz = 0.0, mt = 0.0;
            if (k < count && ((lm[k] >> lane) & 1u)) {
                const double4 c = lc[k];
                const double dx = c.x - bx, dy = c.y - by, dz = c.z - bz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                pair_adjoint<kDamp, double>(dx, dy, dz, r2, c.w, lax, lay, laz, vx, vy, vz, mt);
            }
            gx -= vx; gy -= vy; gz -= vz;
            v[4 * j] = vx; v[4 * j + 1] = vy; v[4 * j + 2] = vz; v[4 * j + 3] = mt;
        }
        const double z = warp_transpose_sum32(v, lane);
        scatter_adj8(adj_node, adj_leaf, lr, k0, count, z, lane);
    }
}

template <bool kDamp, bool kPot>
__device__ inline void force_list_f64(const double4 *lc, const uint32_t *lm, int count, int lane, double bx,
                                      double by, double bz, double &ax, double &ay, double &az, double &pot) {
#pragma unroll 2
    for (int k = 0; k < count; k++) {
        const uint32_t m = lm[k];
        if (!((m >> lane) & 1u)) continue;
        const double4 c = lc[k];
        const double dx = c.x - bx, dy = c.y - by, dz = c.z - bz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double d = sqrt(r2);
        const double inv = 1.0 / d;
        double f;
        if constexpr (kDamp) f = c.w * inv / (r2 + exp(-d));
        else f = c.w * inv * inv * inv;
        ax = fma(f, dx, ax); ay = fma(f, dy, ay); az = fma(f, dz, az);
        if constexpr (kPot) pot += c.w * inv;
    }
}

template <bool kFp64, bool kDamp, bool kPot, bool kAdj, class Sm>
__device__ inline void flush_list(Sm &s, int count, int lane, const WalkArgs &a, const double4 &b, float px, float py,
                                  float pz, double lax, double lay, double laz, float &fax, float &fay, float &faz,
                                  double &dax, double &day, double &daz, double &dpot, uint32_t &cnt) {
    const uint32_t bit = 1u << lane;
    if constexpr (kAdj) {
        if constexpr (kFp64)
            adj_list_f64<kDamp>(s.lc, s.lm, s.lr, count, lane, b.x, b.y, b.z, lax, lay, laz, dax, day, daz, a.adj_node,
                                a.adj_leaf);
        else
            adj_list_f32<kDamp>(s.lc, s.lm, s.lr, count, lane, px, py, pz, (float)lax, (float)lay, (float)laz, fax, fay,
                                faz, a.adj_node, a.adj_leaf);
    } else {
        if constexpr (kFp64) force_list_f64<kDamp, kPot>(s.lc, s.lm, count, lane, b.x, b.y, b.z, dax, day, daz, dpot);
        else force_pairs_f32<kDamp, true>(s.lp, s.lm, count, bit, px, py, pz, fax, fay, faz);
    }
    if (a.counts) cnt += count_list(s.lm, count, bit);
}

template <bool kFp64, bool kDamp, bool kPot, bool kAdj, bool kStats>
__global__ void __launch_bounds__(kWalkMaxWarps * 32) k_walk(WalkArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    griddep();
    using Sm = WarpSmem<kFp64>;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    Sm &s = reinterpret_cast<Sm *>(smem_raw)[wid];
    const Tree &t = a.t;
    const uint32_t n = t.n;
    const bool single = a.single != 0;
    const float theta_f = __double2float_rn(a.theta);
    const double theta = single ? (double)theta_f : a.theta;
    // relative width of the FP64 form's group-level band: its own rounding, or
    // the FLOAT build's (~6.3 float ulps of (side/theta)^2)
    const double grp_rel = single ? 1e-6 : 1e-12;
    const double S1 = t.sc->root_side;
    int2 *gspill = a.spill + (size_t)(blockIdx.x * (blockDim.x >> 5) + wid) * a.spill_cap;
    const unsigned FULL = 0xffffffffu;
    const uint32_t lt = (1u << lane) - 1u;

    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(&t.sc->group_counter, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= a.n_groups) break;

        uint32_t g0, gcount;
        int root = 0;
        double S = S1;
        if (a.groups) {
            const int4 gr = a.groups[g];
            g0 = (uint32_t)gr.x;
            gcount = (uint32_t)gr.y;
            root = a.sys_root_node[gr.z];
            S = a.sys_root[4 * (size_t)gr.z + 3];
        } else {
            g0 = g * 32;
            gcount = min(32u, n - g0);
            root = n >= 2 ? 0 : -1;
        }
        const double s_theta = S / theta;
        const uint32_t j = g0 + lane;
        const bool valid = (uint32_t)lane < gcount;
        const double4 b = t.body[valid ? j : g0];
        const uint32_t vmask = __ballot_sync(FULL, valid);
        // adjoint mode: this particle's cotangent dL/da
        double lax = 0.0, lay = 0.0, laz = 0.0;
        if constexpr (kAdj) {
            if (valid) {
                const size_t u3 = 3 * (size_t)t.sidx[j];
                if constexpr (kFp64) { lax = a.lamd[u3]; lay = a.lamd[u3 + 1]; laz = a.lamd[u3 + 2]; }
                else { lax = a.lamf[u3]; lay = a.lamf[u3 + 1]; laz = a.lamf[u3 + 2]; }
            }
        }

        // Reference point: centre of the group's bounding box.
        const double rx = 0.5 * (warp_min(b.x) + warp_max(b.x));
        const double ry = 0.5 * (warp_min(b.y) + warp_max(b.y));
        const double rz = 0.5 * (warp_min(b.z) + warp_max(b.z));
        const float px = (float)(b.x - rx), py = (float)(b.y - ry), pz = (float)(b.z - rz);
        // what the FP32 offsets left out (the forward near list adds it back)
        const float plx = lo_part(b.x - rx, px), ply = lo_part(b.y - ry, py), plz = lo_part(b.z - rz, pz);
        // Error band of the FP32 opening test. With u = 2^-24 and Pm the largest
        // |offset| from the reference point in the group, every lane has
        // |r2_f32 - r2| <= 7.1u r2 + 7u Pm sqrt(r2) and |q_f32 - q| <= 1.01u q;
        // outside |r2 - q| <= 32u q + 20u Pm sqrt(q), and for r2 > (64u Pm)^2,
        // the FP32 decision equals the exact one. Inside, the lane re-tests in FP64.
        const float pm_g = warp_maxf(fmaxf(fabsf(px), fmaxf(fabsf(py), fabsf(pz))));
        const float pm_tol = kTolPm * pm_g;
        const float tiny = (kTiny * pm_g) * (kTiny * pm_g);
        const float near_r2 = (pm_g * 0x1p-9f) * (pm_g * 0x1p-9f);
        // Group bounding box of the offsets (lanes past n repeat lane 0): FP32
        // for the MIXED form, FP64 for the FP64 form (group-level test only).
        float lox = 0.f, hix = 0.f, loy = 0.f, hiy = 0.f, loz = 0.f, hiz = 0.f;
        double dlox = 0.0, dhix = 0.0, dloy = 0.0, dhiy = 0.0, dloz = 0.0, dhiz = 0.0, dpm = 0.0;
        if constexpr (kFp64) {
            dlox = warp_min(b.x) - rx; dhix = warp_max(b.x) - rx;
            dloy = warp_min(b.y) - ry; dhiy = warp_max(b.y) - ry;
            dloz = warp_min(b.z) - rz; dhiz = warp_max(b.z) - rz;
            dpm = fmax(fmax(fmax(-dlox, dhix), fmax(-dloy, dhiy)), fmax(-dloz, dhiz));
        } else {
            lox = warp_minf(px); hix = warp_maxf(px);
            loy = warp_minf(py); hiy = warp_maxf(py);
            loz = warp_minf(pz); hiz = warp_maxf(pz);
        }

        if (lane == 0) {
            s.gc.ref[0] = rx; s.gc.ref[1] = ry; s.gc.ref[2] = rz;
            s.gc.S = S; s.gc.s_theta = s_theta;
            s.gc.box[0] = lox; s.gc.box[1] = hix; s.gc.box[2] = loy;
            s.gc.box[3] = hiy; s.gc.box[4] = loz; s.gc.box[5] = hiz;
            s.gc.pm_tol = pm_tol; s.gc.tiny = tiny; s.gc.near_r2 = near_r2;
            if constexpr (kStats)
                for (int q = 0; q < 6; q++) s.gc.st[q] = 0u;
        }
        float fax = 0.f, fay = 0.f, faz = 0.f;
        double dax = 0.0, day = 0.0, daz = 0.0, dpot = 0.0;
        uint32_t cnt = 0, nint = 0, nfallback = 0;
        int top = 0, list_top = 0, full_top = 0, near_top = 0;
        uint32_t spill_top = 0;
        bool failed = false;
        if (root >= 0) {
            if (lane == 0) s.stack[0] = make_int2(root, (int)vmask);
            top = 1;
        }
        __syncwarp();

        while (top > 0 || spill_top > 0) {
            if (top == 0) spill_in(s, top, spill_top, gspill, lane);
            const int cntt = min(top, 32);
            const int base = top - cntt;
            top = base;
            if (kStats && lane == 0) { s.gc.st[0] += cntt; s.gc.st[1] += 1u; }

            // ---- stage: lane k takes stack entry k
            bool is_int = false;
            int4 ch0 = make_int4(0, 0, 0, 0), ch1 = make_int4(0, 0, 0, 0);
            uint32_t reach = 0;
            int nch = 0, ref = 0;
            double cx = 0, cy = 0, cz = 0, m = 0, so = 0;
            if (lane < cntt) {
                const int2 e = s.stack[base + lane];
                ref = e.x;
                reach = (uint32_t)e.y;
                if (ref >= 0) {
                    const double4 nd = t.onode[ref];
                    const int meta = t.ometa[ref];
                    cx = nd.x; cy = nd.y; cz = nd.z; m = nd.w;
                    nch = meta_nchild(meta);
                    so = exp2_neg(meta_level(meta));  // 2^-level
                    const int4 *cp = reinterpret_cast<const int4 *>(t.ochild + 8 * (size_t)ref);
                    ch0 = cp[0];
                    ch1 = cp[1];
                    is_int = true;
                } else {
                    const double4 bd = t.body[~ref];
                    cx = bd.x; cy = bd.y; cz = bd.z; m = bd.w;
                    const uint32_t own = (uint32_t)(~ref) - g0;  // a leaf of this group: not its own lane
                    if (own < 32u) reach &= ~(1u << own);
                }
            }
            float fcx = 0.f, fcy = 0.f, fcz = 0.f;
            if constexpr (!kFp64) {
                fcx = (float)(cx - s.gc.ref[0]); fcy = (float)(cy - s.gc.ref[1]); fcz = (float)(cz - s.gc.ref[2]);
            }

            // ---- group-level test, one node per lane: when every point of the
            // group's box (widened by twice the FP32 error band) lies beyond the
            // opening radius side/theta, no lane opens the node; when every point
            // lies within it, every lane that reached it opens it. Only the
            // remaining nodes are decided lane by lane below.
            uint32_t my_open = 0;
            bool mixed = false;
            float r2box = 0.f;  // squared distance of the node from the group's box (MIXED form)
            float qf = 0.f, band = 0.f;  // (side/theta)^2 in FP32 and the half-width of its error band
            if (is_int) {
                if constexpr (kFp64) {
                    const double sq = s.gc.S * so / theta;
                    const double qd = sq * sq;
                    const double ox = cx - s.gc.ref[0], oy = cy - s.gc.ref[1], oz = cz - s.gc.ref[2];
                    const double ax_ = fmax(fmax(dlox - ox, ox - dhix), 0.0), ay_ = fmax(fmax(dloy - oy, oy - dhiy), 0.0),
                                 az_ = fmax(fmax(dloz - oz, oz - dhiz), 0.0);
                    const double bx_ = fmax(fabs(ox - dlox), fabs(ox - dhix)), by_ = fmax(fabs(oy - dloy), fabs(oy - dhiy)),
                                 bz_ = fmax(fabs(oz - dloz), fabs(oz - dhiz));
                    const double r2min = ax_ * ax_ + ay_ * ay_ + az_ * az_;
                    const double r2max = bx_ * bx_ + by_ * by_ + bz_ * bz_;
                    const double tol = grp_rel * (qd + dpm * sq) + 1e-300;
                    if (r2min - qd > tol) my_open = 0;
                    else if (qd - r2max > tol) my_open = reach;
                    else mixed = true;
                } else {
                    const double sqd = s.gc.s_theta * so;
                    qf = (float)(sqd * sqd);
                    band = fmaf(s.gc.pm_tol, (float)sqd, kTolRel * qf);
                    const float tol = 2.f * band;
                    const float ax_ = fmaxf(fmaxf(s.gc.box[0] - fcx, fcx - s.gc.box[1]), 0.f), ay_ = fmaxf(fmaxf(s.gc.box[2] - fcy, fcy - s.gc.box[3]), 0.f),
                                az_ = fmaxf(fmaxf(s.gc.box[4] - fcz, fcz - s.gc.box[5]), 0.f);
                    const float bx_ = fmaxf(fabsf(fcx - s.gc.box[0]), fabsf(fcx - s.gc.box[1])), by_ = fmaxf(fabsf(fcy - s.gc.box[2]), fabsf(fcy - s.gc.box[3])),
                                bz_ = fmaxf(fabsf(fcz - s.gc.box[4]), fabsf(fcz - s.gc.box[5]));
                    const float r2min = fmaf(az_, az_, fmaf(ay_, ay_, ax_ * ax_));
                    const float r2max = fmaf(bz_, bz_, fmaf(by_, by_, bx_ * bx_));
                    r2box = r2min;
                    if (r2min <= 4.f * s.gc.tiny) mixed = true;
                    else if (r2min - qf > tol) my_open = 0;
                    else if (qf - r2max > tol) my_open = reach;
                    else mixed = true;
                }
            }

            // ---- decide the mixed nodes of the tile, lane by lane
            const uint32_t intm = __ballot_sync(FULL, mixed);
            if (kStats && lane == 0) s.gc.st[2] += __popc(intm);
            if (intm) {
                if constexpr (kFp64) {
                    s.tc[lane] = make_double4(cx, cy, cz, s.gc.S * so);
                    s.tr[lane] = make_int2((int)reach, ref);
                    __syncwarp();
                }
                if constexpr (kFp64) {
                    // the FP64 form decides every mixed node with the reference's own test
                    uint32_t mm = intm;
                    while (mm) {
                        const int k = __ffs(mm) - 1;
                        mm &= mm - 1;
                        const double4 c = s.tc[k];
                        const uint32_t rk = (uint32_t)s.tr[k].x;
                        const bool open = ref_open(single, c.x, c.y, c.z, b.x, b.y, b.z, c.w, theta, theta_f);
                        const uint32_t om = __ballot_sync(FULL, open) & rk;
                        if (lane == k) my_open = om;
                    }
                } else {
                    // The mixed nodes, compacted into pairs, are decided two per round
                    // with packed FP32 arithmetic (the same roundings as the scalar
                    // expressions: dx = c.x + (-px), r2 = fma(dz, dz, fma(dy, dy, dx dx)),
                    // d = r2 + (-q)). Lane 0 stores each pair's open masks over the
                    // pair's first two words; each mixed lane then reads its own.
                    const int nmix = __popc(intm);
                    const int mpos = __popc(intm & lt);
                    if (mixed) {
                        float *e = s.mx + 16 * (mpos >> 1) + (mpos & 1);
                        e[0] = fcx; e[2] = fcy; e[4] = fcz; e[6] = -qf;
                        e[8] = band; e[10] = __uint_as_float(reach); e[12] = __int_as_float(ref);
                    }
                    if (lane == 0 && (nmix & 1)) {
                        // pad an odd count with an entry no lane reached
                        float *e = s.mx + 16 * (nmix >> 1) + 1;
                        e[0] = 0.f; e[2] = 0.f; e[4] = 0.f; e[6] = 0.f;
                        e[8] = 0.f; e[10] = 0.f; e[12] = 0.f;
                    }
                    __syncwarp();
                    const float tiny_ = s.gc.tiny;
                    const uint64_t npx = f2pack(-px, -px), npy = f2pack(-py, -py), npz = f2pack(-pz, -pz);
                    const uint32_t bit = 1u << lane;
                    for (int k = 0; k < nmix; k += 2) {
                        float *pr = s.mx + 8 * k;
                        const float4 A = *reinterpret_cast<const float4 *>(pr);      // x0 x1 y0 y1
                        const float4 B = *reinterpret_cast<const float4 *>(pr + 4);  // z0 z1 -q0 -q1
                        const float4 C = *reinterpret_cast<const float4 *>(pr + 8);  // band0 band1 reach0 reach1
                        const uint64_t dx = f2add(f2pack(A.x, A.y), npx);
                        const uint64_t dy = f2add(f2pack(A.z, A.w), npy);
                        const uint64_t dz = f2add(f2pack(B.x, B.y), npz);
                        const uint64_t r2 = f2fma(dz, dz, f2fma(dy, dy, f2mul(dx, dx)));
                        const uint64_t dd = f2add(r2, f2pack(B.z, B.w));
                        float r21, r22, d1, d2;
                        f2unpack(r2, r21, r22);
                        f2unpack(dd, d1, d2);
                        const uint32_t rk1 = __float_as_uint(C.z), rk2 = __float_as_uint(C.w);
                        bool open1 = d1 < 0.f, open2 = d2 < 0.f;
                        const bool amb1 = (rk1 & bit) && (fabsf(d1) <= C.x || r21 <= tiny_);
                        const bool amb2 = (rk2 & bit) && (fabsf(d2) <= C.y || r22 <= tiny_);
                        if (__any_sync(FULL, amb1 || amb2)) {
                            const float2 R = *reinterpret_cast<const float2 *>(pr + 12);  // ref0 ref1
                            if (amb1) {
                                const int node = __float_as_int(R.x);
                                const double4 nd = t.onode[node];
                                const double side = s.gc.S * exp2_neg(meta_level(t.ometa[node]));
                                open1 = ref_open(single, nd.x, nd.y, nd.z, b.x, b.y, b.z, side, theta, theta_f);
                                nfallback++;
                            }
                            if (amb2) {
                                const int node = __float_as_int(R.y);
                                const double4 nd = t.onode[node];
                                const double side = s.gc.S * exp2_neg(meta_level(t.ometa[node]));
                                open2 = ref_open(single, nd.x, nd.y, nd.z, b.x, b.y, b.z, side, theta, theta_f);
                                nfallback++;
                            }
                        }
                        const uint32_t om1 = __ballot_sync(FULL, open1) & rk1;
                        const uint32_t om2 = __ballot_sync(FULL, open2) & rk2;
                        // every lane has read the pair before the ballots complete
                        if (lane == 0) *reinterpret_cast<uint2 *>(pr) = make_uint2(om1, om2);
                    }
                    __syncwarp();
                    if (mixed) my_open = __float_as_uint(s.mx[16 * (mpos >> 1) + (mpos & 1)]);
                }
                __syncwarp();
            }

            // ---- accepted bodies -> interaction list (compacted across lanes).
            // MIXED: a body closer to the group's box than 2^-9 of the group's
            // extent would lose too many bits in FP32 offsets (and could give a
            // zero r^2); it goes to the near list, whose offsets are taken in FP64.
            const uint32_t accm = reach & ~my_open;
            nint += __popc(accm);
            bool near = false;
            if constexpr (!kFp64) {
                if (accm) {
                    if (!is_int) {  // internal nodes have it from the group test
                        const float ax_ = fmaxf(fmaxf(s.gc.box[0] - fcx, fcx - s.gc.box[1]), 0.f),
                                    ay_ = fmaxf(fmaxf(s.gc.box[2] - fcy, fcy - s.gc.box[3]), 0.f),
                                    az_ = fmaxf(fmaxf(s.gc.box[4] - fcz, fcz - s.gc.box[5]), 0.f);
                        r2box = fmaf(az_, az_, fmaf(ay_, ay_, ax_ * ax_));
                    }
                    near = r2box < s.gc.near_r2;
                }
            }
            if constexpr (!kFp64 && !kAdj) {
                // entries every lane of the group takes go to a list without masks
                const bool take = accm != 0 && !near;
                const bool all = take && accm == vmask;
                const uint32_t fmk = __ballot_sync(FULL, all);
                const uint32_t pmk = __ballot_sync(FULL, take && !all);
                const float gmf = (float)(kG * m);
                if (all) {
                    put_pair_entry(s.lf, full_top + __popc(fmk & lt), fcx, fcy, fcz, gmf);
                } else if (take) {
                    const int pos = list_top + __popc(pmk & lt);
                    put_pair_entry(s.lp, pos, fcx, fcy, fcz, gmf);
                    s.lm[pos] = accm;
                }
                full_top += __popc(fmk);
                list_top += __popc(pmk);
                if (kStats && lane == 0) s.gc.st[3] += __popc(fmk) + __popc(pmk);
            } else {
                const uint32_t am = __ballot_sync(FULL, accm != 0 && !near);
                if (accm && !near) {
                    const int pos = list_top + __popc(am & lt);
                    if constexpr (kFp64) s.lc[pos] = make_double4(cx, cy, cz, kG * m);
                    else s.lc[pos] = make_float4(fcx, fcy, fcz, (float)(kG * m));
                    s.lm[pos] = accm;
                    if constexpr (kAdj) s.lr[pos] = ref;
                }
                list_top += __popc(am);
                if (kStats && lane == 0) s.gc.st[3] += __popc(am);
            }
            if constexpr (!kFp64 && !kAdj) {
                // forward: near bodies collect in their own paired list, offsets as hi + lo
                const uint32_t nmk = __ballot_sync(FULL, near);
                if (nmk) {
                    if (near) {
                        const int pos = near_top + __popc(nmk & lt);
                        const double ox = cx - s.gc.ref[0], oy = cy - s.gc.ref[1], oz = cz - s.gc.ref[2];
                        put_pair_entry(s.np.hi, pos, fcx, fcy, fcz, (float)(kG * m));
                        put_pair_entry(s.np.lo, pos, lo_part(ox, fcx), lo_part(oy, fcy), lo_part(oz, fcz), 0.f);
                        s.nm[pos] = accm;
                    }
                    near_top += __popc(nmk);
                    if (kStats && lane == 0) s.gc.st[4] += __popc(nmk);
                }
            } else if constexpr (!kFp64) {
                const uint32_t nmk = __ballot_sync(FULL, near);
                if (nmk) {
                    if (near) {
                        const int pos = __popc(nmk & lt);
                        s.nc[pos] = make_double4(cx, cy, cz, kG * m);
                        s.nm[pos] = accm;
                        s.nr[pos] = ref;
                    }
                    __syncwarp();
                    adj_near_f32<kDamp>(s.nc, s.nm, s.nr, __popc(nmk), lane, b.x, b.y, b.z, (float)lax, (float)lay,
                                        (float)laz, fax, fay, faz, a.adj_node, a.adj_leaf);
                    if (a.counts) cnt += count_list(s.nm, __popc(nmk), 1u << lane);
                    if (kStats && lane == 0) s.gc.st[4] += __popc(nmk);
                    __syncwarp();
                }
            }

            // ---- children of opened nodes -> stack
            // exclusive prefix of the child counts (0..8) from four independent ballots of their bits
            const int myn = my_open ? nch : 0;
            const uint32_t q0 = __ballot_sync(FULL, myn & 1), q1 = __ballot_sync(FULL, myn & 2),
                           q2 = __ballot_sync(FULL, myn & 4), q3 = __ballot_sync(FULL, myn & 8);
            const int pre = __popc(q0 & lt) + 2 * __popc(q1 & lt) + 4 * __popc(q2 & lt) + 8 * __popc(q3 & lt);
            const int total = __popc(q0) + 2 * __popc(q1) + 4 * __popc(q2) + 8 * __popc(q3);
            if (total > 0) {
                if (top + total > kStackCap) {
                    if (!spill_out(s, top, spill_top, gspill, a.spill_cap, lane)) {
                        failed = true;
                        break;
                    }
                }
                int2 *dst = s.stack + top + pre;
                const int om = (int)my_open;
                if (myn > 0) dst[0] = make_int2(ch0.x, om);
                if (myn > 1) dst[1] = make_int2(ch0.y, om);
                if (myn > 2) dst[2] = make_int2(ch0.z, om);
                if (myn > 3) dst[3] = make_int2(ch0.w, om);
                if (myn > 4) dst[4] = make_int2(ch1.x, om);
                if (myn > 5) dst[5] = make_int2(ch1.y, om);
                if (myn > 6) dst[6] = make_int2(ch1.z, om);
                if (myn > 7) dst[7] = make_int2(ch1.w, om);
                top += total;
                if (kStats && lane == 0) s.gc.st[5] = max(s.gc.st[5], (uint32_t)(top + (int)spill_top));
            }
            __syncwarp();

            // ---- forces once a list is long enough
            if (list_top >= kListFlush) {
                flush_list<kFp64, kDamp, kPot, kAdj>(s, list_top, lane, a, b, px, py, pz, lax, lay, laz, fax, fay, faz,
                                                      dax, day, daz, dpot, cnt);
                list_top = 0;
                __syncwarp();
            }
            if constexpr (!kFp64 && !kAdj) {
                if (full_top >= kListFlush) {
                    force_pairs_f32<kDamp, false>(s.lf, nullptr, full_top, 0u, px, py, pz, fax, fay, faz);
                    cnt += full_top;
                    full_top = 0;
                    __syncwarp();
                }
                if (near_top >= kListFlush) {
                    force_pairs_f32<kDamp, true, true>(s.np.hi, s.nm, near_top, 1u << lane, px, py, pz, fax, fay, faz,
                                                       s.np.lo, plx, ply, plz);
                    if (a.counts) cnt += count_list(s.nm, near_top, 1u << lane);
                    near_top = 0;
                    __syncwarp();
                }
            }
        }
        if (failed && lane == 0) atomicOr(&t.sc->status, kStatusCapacity);
        if (list_top > 0) {
            flush_list<kFp64, kDamp, kPot, kAdj>(s, list_top, lane, a, b, px, py, pz, lax, lay, laz, fax, fay, faz,
                                                  dax, day, daz, dpot, cnt);
        }
        if constexpr (!kFp64 && !kAdj) {
            if (full_top > 0) {
                force_pairs_f32<kDamp, false>(s.lf, nullptr, full_top, 0u, px, py, pz, fax, fay, faz);
                cnt += full_top;
            }
            if (near_top > 0) {
                force_pairs_f32<kDamp, true, true>(s.np.hi, s.nm, near_top, 1u << lane, px, py, pz, fax, fay, faz,
                                                   s.np.lo, plx, ply, plz);
                if (a.counts) cnt += count_list(s.nm, near_top, 1u << lane);
            }
        }
        __syncwarp();

        // ---- epilogue: results in the caller's particle order
        double ax, ay, az;
        if constexpr (kFp64) { ax = dax; ay = day; az = daz; }
        else { ax = fax; ay = fay; az = faz; }
        if (valid) {
            const uint32_t ui = t.sidx[j];
            if constexpr (kAdj) {
                if constexpr (kFp64) {
                    a.gdird[3 * (size_t)ui] = ax; a.gdird[3 * (size_t)ui + 1] = ay; a.gdird[3 * (size_t)ui + 2] = az;
                } else {
                    a.gdirf[3 * (size_t)ui] = fax; a.gdirf[3 * (size_t)ui + 1] = fay; a.gdirf[3 * (size_t)ui + 2] = faz;
                }
            } else if constexpr (kFp64) {
                a.accd[3 * (size_t)ui] = ax; a.accd[3 * (size_t)ui + 1] = ay; a.accd[3 * (size_t)ui + 2] = az;
            } else {
                a.accf[3 * (size_t)ui] = fax; a.accf[3 * (size_t)ui + 1] = fay; a.accf[3 * (size_t)ui + 2] = faz;
            }
            if (a.counts) a.counts[ui] = cnt;
            if constexpr (kPot) {
                if (a.pot) a.pot[ui] = -dpot;
            }
        }
        unsigned long long wc = nint;
        for (int o = 16; o; o >>= 1) wc += __shfl_xor_sync(FULL, wc, o);
        uint32_t wf = nfallback;
        for (int o = 16; o; o >>= 1) wf += __shfl_xor_sync(FULL, wf, o);
        double amag = valid ? sqrt(ax * ax + ay * ay + az * az) : 0.0;
        if (!kAdj && a.track_max_acc) amag = warp_max(amag);
        if (lane == 0) {
            atomicAdd(&t.sc->interactions, wc);
            atomicAdd(&t.sc->interactions_total, wc);
            if (wf) atomicAdd(&t.sc->fallback_tests, wf);
            if constexpr (kStats) {
                atomicAdd(&t.sc->walk_entries, (unsigned long long)s.gc.st[0]);
                atomicAdd(&t.sc->walk_tiles, (unsigned long long)s.gc.st[1]);
                atomicAdd(&t.sc->walk_decisions, (unsigned long long)s.gc.st[2]);
                atomicAdd(&t.sc->walk_list, (unsigned long long)s.gc.st[3]);
                if (s.gc.st[4]) atomicAdd(&t.sc->walk_near, (unsigned long long)s.gc.st[4]);
                atomicMax(&t.sc->max_stack, s.gc.st[5]);
            }
            if (!kAdj && a.track_max_acc) atomic_max_nonneg(&t.sc->max_acc_bits, amag);
        }
    }
}

// Potentials (diagnostics) are summed by the FP64 form only. The walk's
// statistics (entries, tiles, decisions, list and near entries, deepest stack)
// are collected by their own instances of the forward kernel (kStats), so that
// the others carry none of that bookkeeping; the adjoint collects none.
template <bool kFp64, bool kStats>
const void *forward_kernel(int damping, bool pot) {
    if constexpr (!kFp64) {
        (void)pot;
        return damping ? (const void *)k_walk<false, true, false, false, kStats>
                       : (const void *)k_walk<false, false, false, false, kStats>;
    } else {
        if (damping)
            return pot ? (const void *)k_walk<true, true, true, false, kStats>
                       : (const void *)k_walk<true, true, false, false, kStats>;
        return pot ? (const void *)k_walk<true, false, true, false, kStats>
                   : (const void *)k_walk<true, false, false, false, kStats>;
    }
}

const void *any_walk_kernel(bool fp64, bool adj, int damping, bool pot, bool stats) {
    if (adj) {
        if (fp64) return damping ? (const void *)k_walk<true, true, false, true, false> : (const void *)k_walk<true, false, false, true, false>;
        return damping ? (const void *)k_walk<false, true, false, true, false> : (const void *)k_walk<false, false, false, true, false>;
    }
    if (fp64) return stats ? forward_kernel<true, true>(damping, pot) : forward_kernel<true, false>(damping, pot);
    return stats ? forward_kernel<false, true>(damping, pot) : forward_kernel<false, false>(damping, pot);
}

}  // namespace

constexpr size_t kLargestWarpSmem =
    sizeof(WarpSmem<true>) > sizeof(WarpSmem<false>) ? sizeof(WarpSmem<true>) : sizeof(WarpSmem<false>);

cudaError_t walk_max_blocks_per_sm(bool fp64, unsigned warps, int *out) {
    const size_t smem = (fp64 ? sizeof(WarpSmem<true>) : sizeof(WarpSmem<false>)) * warps;
    int minblocks = 1 << 30;
    for (int adj = 0; adj < 2; adj++)
        for (int damp = 0; damp < 2; damp++)
            for (int pot = 0; pot < 2 - adj; pot++)
                for (int stats = 0; stats < 2 - adj; stats++) {
                    const void *k = any_walk_kernel(fp64, adj, damp, pot, stats);
                    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)(kLargestWarpSmem * kWalkMaxWarps));
                    if (e != cudaSuccess) return e;
                    int nb = 0;
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, (int)warps * 32, smem);
                    if (e != cudaSuccess) return e;
                    minblocks = nb < minblocks ? nb : minblocks;
                }
    *out = minblocks;
    return cudaSuccess;
}

cudaError_t walk_launch_shape(bool fp64, int device, unsigned warps, unsigned blocks_per_sm, WalkLaunch *out) {
    int maxb = 0;
    cudaError_t e = walk_max_blocks_per_sm(fp64, warps, &maxb);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    if (maxb < 1) maxb = 1;
    const int per_sm = blocks_per_sm ? (int)blocks_per_sm < maxb ? (int)blocks_per_sm : maxb : maxb;
    out->blocks = (unsigned)(sms * per_sm);
    out->warps = warps;
    out->smem = (fp64 ? sizeof(WarpSmem<true>) : sizeof(WarpSmem<false>)) * warps;
    return cudaSuccess;
}

cudaError_t launch_walk(const WalkArgs &a, bool fp64, const WalkLaunch &l, cudaStream_t st) {
    const void *k = any_walk_kernel(fp64, a.adjoint != 0, a.damping, a.pot != nullptr, a.stats != 0);
    unsigned blocks = l.blocks;
    const unsigned need = (a.n_groups + l.warps - 1) / l.warps;
    if (need < blocks) blocks = need ? need : 1;
    WalkArgs args = a;
    void *params[] = {&args};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(l.warps * 32);
    cfg.dynamicSmemBytes = l.smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, k, params);
}

}  // namespace nbody
