// Root cube without allocation (include/nbody_b200_noalloc.h).
//
// Some callers cannot call cudaMalloc: code that runs while a stream is being
// captured into a CUDA graph (allocation is not allowed inside a global
// capture), plug-ins whose host framework owns every byte of device memory,
// and real-time loops that must never block on the allocator. For them this
// file offers the first reduction of the Barnes-Hut step -- the reference's
// root cube, src/main.cpp:889-920 -- over particle arrays they already hold on
// the device, with its scratch (per-tile partial extrema and a completion
// ticket) in a file-scope device array instead of memory from cudaMalloc.
//
// Limits and sharing: the scratch has room for kMaxTiles tiles of kTile
// particles, so n is at most kMaxTiles * kTile (4,194,304); larger n is
// rejected. Every call in a CUDA context uses the same scratch, which keeps
// the last call's partial extrema; the ticket starts at zero when the module
// is loaded and the last block of every call sets it back to zero. Calls that
// overlap on the GPU (different streams, or host threads, at the same time)
// race on the scratch and must be serialised by the caller.
//
// Contexts: each CUDA context that runs this code holds its own instance of
// the array at its own address. The host looks the address up once per
// context, keyed by the context's unique id (cuCtxGetId), so a context created
// after cudaDeviceReset or by the driver API gets a fresh lookup. The kernel
// also compares the address it is given with the array's address in its own
// context and, if they differ, touches nothing and reports it in out[4].
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/nbody_b200.h"
#include "../../include/nbody_b200_noalloc.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr uint32_t kTile = kThreads * kItems;  // particles reduced by one block
constexpr uint32_t kMaxTiles = 1024;
constexpr uint32_t kMaxN = kTile * kMaxTiles;

struct Scratch {
    double partial[kMaxTiles][8];  // per tile: min x,y,z, -max x,y,z, non-finite flag
    unsigned int ticket;
};

static __device__ __align__(256) Scratch g_scratch;

__device__ inline double wmin(double v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void __launch_bounds__(kThreads) k_root_cube_static(const double *__restrict__ pos,
                                                                const double *__restrict__ mass, uint32_t n,
                                                                Scratch *sc, double *__restrict__ out) {
    // The host's address must be this context's instance of the array; if not,
    // nothing is read or written through it.
    if (sc != &g_scratch) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int k = 0; k < 4; k++) out[k] = NAN;
            out[4] = 2.0;
        }
        return;
    }
    __shared__ double s_red[7][kThreads / 32];
    __shared__ bool s_last;
    double v[7] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};
    const uint32_t base = blockIdx.x * kTile;
    for (int r = 0; r < kItems; r++) {
        const uint32_t i = base + r * kThreads + threadIdx.x;
        if (i >= n) break;
        const double x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
        const double m = mass[i];
        if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(m))) v[6] = -1.0;
        v[0] = fmin(v[0], x); v[1] = fmin(v[1], y); v[2] = fmin(v[2], z);
        v[3] = fmin(v[3], -x); v[4] = fmin(v[4], -y); v[5] = fmin(v[5], -z);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < 7; k++) {
        const double r = wmin(v[k]);
        if (lane == 0) s_red[k][wid] = r;
    }
    __syncthreads();
    if (wid == 0) {
        for (int k = 0; k < 7; k++) {
            double r = lane < kThreads / 32 ? s_red[k][lane] : INFINITY;
            r = wmin(r);
            if (lane == 0) sc->partial[blockIdx.x][k] = r;
        }
        if (lane == 0) {
            __threadfence();
            s_last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!s_last || wid != 0) return;
    __threadfence();
    double r[7];
    for (int k = 0; k < 7; k++) {
        double a = INFINITY;
        for (uint32_t b = lane; b < gridDim.x; b += 32) a = fmin(a, __ldcg(&sc->partial[b][k]));
        r[k] = wmin(a);
    }
    if (lane == 0) {
        // every block has taken its ticket: the next call starts from zero
        sc->ticket = 0u;
        if (r[6] < 0.0) {
            // fmin skips NaN, so the extrema would look valid: the cube is poisoned instead
            for (int k = 0; k < 4; k++) out[k] = NAN;
            out[4] = 1.0;
            return;
        }
        const double lo[3] = {r[0], r[1], r[2]}, hi[3] = {-r[3], -r[4], -r[5]};
        for (int k = 0; k < 3; k++) out[k] = (lo[k] + hi[k]) / 2.0;
        const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
        double side;
        if (ex > ey && ex > ez) side = ex + 2.0;
        else if (ey > ex && ey > ez) side = ey + 2.0;
        else side = ez + 2.0;
        out[3] = side;
        out[4] = 0.0;
    }
}

// Driver queries for the calling thread's current context, resolved through
// the runtime so that the library needs no link against libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_fns_once;

void resolve_driver_fns() {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
}

// Unique id of the calling thread's current context, or false when no live
// context is current (a fresh thread, or right after a device reset).
bool current_context_id(unsigned long long *id) {
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of g_scratch in each context seen so far (most recent first).
constexpr int kMaxContexts = 64;
struct CtxAddr {
    unsigned long long id;
    Scratch *addr;
};
CtxAddr g_addr[kMaxContexts];
int g_naddr = 0;
std::mutex g_mu;

// Set-up for the current context: the device address of g_scratch, looked up
// with cudaGetSymbolAddress the first time a context is seen.
int scratch_for_current_context(Scratch **ptr) {
    std::call_once(g_fns_once, resolve_driver_fns);
    if (!g_ctx_get_current || !g_ctx_get_id) return NBODY_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return NBODY_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned long long id = 0;
    const bool have_ctx = current_context_id(&id);
    if (have_ctx) {
        for (int i = 0; i < g_naddr; i++)
            if (g_addr[i].id == id) {
                *ptr = g_addr[i].addr;
                return NBODY_OK;
            }
    }
    // First call in this context. The lookup also makes the runtime bind (and,
    // after a reset, re-create) the device's context when none is current.
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return NBODY_ERR_CUDA;
    }
    if (!have_ctx && !current_context_id(&id)) return NBODY_ERR_CUDA;
    const int slot = g_naddr < kMaxContexts ? g_naddr++ : kMaxContexts - 1;
    for (int i = slot; i > 0; i--) g_addr[i] = g_addr[i - 1];
    g_addr[0] = CtxAddr{id, static_cast<Scratch *>(p)};
    *ptr = static_cast<Scratch *>(p);
    return NBODY_OK;
}

}  // namespace

extern "C" uint32_t nbody_root_cube_noalloc_max_n(void) { return kMaxN; }

extern "C" int nbody_root_cube_noalloc(const double *d_pos, const double *d_mass, uint32_t n, double *d_out,
                                       void *stream) {
    if (n == 0 || !d_pos || !d_mass || !d_out) return NBODY_ERR_INVALID;
    if (n > kMaxN) return NBODY_ERR_INVALID;  // scratch holds kMaxTiles tiles of kTile particles
    Scratch *sc = nullptr;
    int rc = scratch_for_current_context(&sc);
    if (rc != NBODY_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    k_root_cube_static<<<tiles, kThreads, 0, st>>>(d_pos, d_mass, n, sc, d_out);
    return cudaGetLastError() == cudaSuccess ? NBODY_OK : NBODY_ERR_CUDA;
}
