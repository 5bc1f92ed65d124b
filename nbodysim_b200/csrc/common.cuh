// Shared definitions of the nbody_b200 kernels (sm_100a).
//
// Data layout in HBM (capacity `cap` particles, grown on demand, never freed
// per step):
//   user order    pos, vel  : double[3*cap] (AoS, the host layout)
//                 mass      : double[cap]
//                 acc       : float[3*cap] (MIXED) or double[3*cap] (FP64)
//   sort          key1/idx  : u64/u32 [cap] x2 (ping-pong), key2/key3 u64[cap] (deep keys)
//   sorted bodies body      : double4[cap] = (x, y, z, m) in Morton order
//   binary tree   bleft/bright/bparent : i32[cap], bdelta u8..i32[cap], leaf_bparent i32[cap]
//   octree        onode     : double4[cap] = (com.x, com.y, com.z, mass)
//                 ochild    : i32[8*cap]  (>= 0 internal node, < 0 leaf ~sorted index)
//                 ometa     : i32[cap]    level | nchild << 8
//                 oparent   : i32[cap], leaf_oparent : i32[cap], ocount : u32[cap]
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

namespace nbody {

// Programmatic dependent launch (sm_90 and later). The kernels of a force pass
// and a step are launched with launch_pdl: the next kernel in the stream may be
// scheduled while the previous one drains, and every such kernel first waits in
// griddep_wait() until the previous kernel has completed and its memory is
// visible (so it reads nothing of it too early), then lets the kernel after it
// be scheduled (griddep_launch). Launched without the attribute, both are no-ops.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void griddep() {
    griddep_wait();
    griddep_launch();
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr double kG = 6.67384e-11;  // src/main.cpp:322
constexpr int kLevelsPerWord = 21;  // 63 key bits per 64-bit word, 3 bits per octree level
constexpr int kMaxWords = 3;        // up to 63 levels below the root cube
constexpr int kMaxLevels = kLevelsPerWord * kMaxWords;

// Device status bits (OR-ed by kernels, read by the host after a pass).
enum : uint32_t {
    kStatusNonFinite = 1u << 0,
    kStatusCoincident = 1u << 1,
    kStatusCapacity = 1u << 2,
    kStatusDeepGroup = 1u << 3,  // a group of equal 42-level keys needed a third key word
    kStatusSortStall = 1u << 4,  // a radix-sort look-back gave up waiting (never expected)
};

// Pairs of neighbouring keys are binned by the sort passes that separate them:
// 1-8 passes cover the first 63-bit key word, 9-16 also the second; bin 17 is a
// pair equal over both words.
constexpr int kPassBins = 18;
__host__ __device__ inline int passes_for_bits(uint32_t bits) {
    return bits <= 63 ? (int)(bits + 7) / 8 : bits <= 126 ? 8 + (int)(bits - 63 + 7) / 8 : kPassBins - 1;
}

struct DevScalars {
    double root_center[3];
    double root_side;
    double bbox_min[3];
    double bbox_max[3];
    unsigned long long interactions;
    unsigned long long interactions_total;  // summed over the steps of one API call
    unsigned long long walk_entries;        // node entries the walk warps tested (union lists)
    unsigned long long walk_tiles;          // stack tiles the walk warps staged
    unsigned long long walk_decisions;      // internal nodes decided by a warp
    unsigned long long walk_list;           // bodies entered in the warps' interaction lists
    unsigned long long walk_near;           // bodies taken with FP64 offsets (near the group box)
    uint32_t status;
    uint32_t n_onodes;
    uint32_t depth;
    uint32_t max_stack;
    uint32_t fallback_tests;
    uint32_t group_counter;
    uint32_t ticket;          // last-block tickets of reductions
    uint32_t deep_groups;
    uint32_t word_ties;       // the last build's planned sort left a long run of equal neighbours (the full sort ran)
    uint32_t tie_runs;        // short runs of equal neighbours the last build sorted in place
    uint32_t max_prefix_bits; // deepest split of the last build: key bits that separate every
                              // pair of neighbours (the longest common prefix + 1)
    uint32_t pair_passes[kPassBins];  // the last build's pairs of neighbours by the 8-bit sort passes
                                      // that separate them (kPassBins - 1: more than two key words)
    unsigned long long max_acc_bits;  // max |a| (non-negative double as ordered bits)
    unsigned long long max_vel_bits;  // max |v|
    double dt_used;
    // MIXED adjoint: the FP32 cotangents are the FP64 ones times 2^-e, with 2^e
    // the power of two that brings the largest into [0.5, 1); results are
    // multiplied back by lam_scale = 2^e in FP64.
    unsigned long long lam_max_bits;  // max |cotangent| (non-negative double as ordered bits)
    double lam_scale;
    double diag[16];          // kinetic, potential, momentum[3], L[3], mass, m*x[3]
};

struct Tree {
    uint32_t n;
    const double4 *body;       // sorted (x, y, z, m)
    const uint32_t *sidx;      // sorted position -> user index
    const double4 *onode;      // internal nodes (com, mass)
    const int32_t *ochild;     // 8 per node
    const int32_t *ometa;      // level | nchild << 8
    DevScalars *sc;
};

__host__ __device__ inline int meta_level(int32_t m) { return m & 0xff; }
__host__ __device__ inline int meta_nchild(int32_t m) { return (m >> 8) & 0xf; }
__host__ __device__ inline int meta_ninternal(int32_t m) { return (m >> 12) & 0xf; }  // children that are nodes

// Exactly 2^-L for 0 <= L <= 1022 (cell sides halve exactly level by level).
__device__ inline double exp2_neg(int L) { return __longlong_as_double((long long)(1023 - L) << 52); }

// Non-negative doubles compare like their bit patterns.
__device__ inline void atomic_max_nonneg(unsigned long long *a, double v) {
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

__device__ inline double warp_min(double v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline double warp_max(double v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline float warp_minf(float v) {
    for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline float warp_maxf(float v) {
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline double warp_sum(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace nbody
