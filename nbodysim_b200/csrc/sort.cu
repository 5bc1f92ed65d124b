// LSD radix sort of (u64 key, u32 index) pairs, one kernel per 8-bit pass.
//
// The global digit counts of every pass do not depend on the order of the
// keys, so one kernel computes them for all passes up front. Each pass then
// is a single kernel: a block takes the next tile (4096 keys) in ticket order,
// ranks its keys stably (per warp, 16 rounds of 32 keys; the lanes that share
// a digit are found with eight ballots, one per digit bit),
// publishes its per-digit count, adds the counts of all earlier tiles by
// decoupled look-back (a tile only ever waits for tiles that started before
// it, so the wait always ends; it is still bounded, and a timeout is reported
// as an error), and scatters: the tile is first laid out in digit order in
// shared memory, so that each digit's run goes out in coalesced writes.
#include "sort.cuh"
#include "common.cuh"

namespace nbody {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr uint32_t kTile = kThreads * kItems;
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kValue = (1u << 30) - 1;
constexpr uint32_t kSpinLimit = 1u << 20;

// Global digit histograms: pa passes of wa (slots slot_a..), pb of wb (slot_b..)
// and, with wc non-null, the two bytes of wc (slot_c, slot_c + 1). Shared
// counters are indexed by the pass's position in that list.
__global__ void k_hist(const uint64_t *__restrict__ wa, int pa, int slot_a, const uint64_t *__restrict__ wb, int pb,
                       int slot_b, const uint32_t *__restrict__ wc, int slot_c, uint32_t n,
                       uint32_t *__restrict__ ghist, const uint32_t *run_if) {
    griddep();
    __shared__ uint32_t s_h[18 * 256];
    if (run_if && *run_if == 0u) return;
    const int pc = wc ? 2 : 0, np = pa + pb + pc;
    for (int i = threadIdx.x; i < np * 256; i += blockDim.x) s_h[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (pa > 0) {
            const uint64_t a = wa[i];
            for (int k = 0; k < pa; k++) atomicAdd(&s_h[k * 256 + ((a >> digit_shift(pa, k)) & 255u)], 1u);
        }
        if (pb > 0) {
            const uint64_t b = wb[i];
            for (int k = 0; k < pb; k++) atomicAdd(&s_h[(pa + k) * 256 + ((b >> digit_shift(pb, k)) & 255u)], 1u);
        }
        if (pc) {
            const uint32_t c = wc[i];
            atomicAdd(&s_h[(pa + pb) * 256 + (c & 255u)], 1u);
            atomicAdd(&s_h[(pa + pb + 1) * 256 + ((c >> 8) & 255u)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np * 256; i += blockDim.x) {
        const int k = i >> 8;
        const int slot = k < pa ? slot_a + k : k < pa + pb ? slot_b + (k - pa) : slot_c + (k - pa - pb);
        if (s_h[i]) atomicAdd(&ghist[slot * 256 + (i & 255)], s_h[i]);
    }
}

// Zeroes `words` 32-bit words (16-byte aligned), four per thread and step.
__global__ void k_zero_words(uint32_t *__restrict__ p, size_t words) {
    griddep();
    const size_t q = words / 4, stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += stride)
        reinterpret_cast<uint4 *>(p)[i] = make_uint4(0u, 0u, 0u, 0u);
    for (size_t i = 4 * q + blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) p[i] = 0u;
}

// Exclusive scan of each pass's 256 counts (one block per pass, in the order of k_hist).
__global__ void k_hist_scan(uint32_t *__restrict__ ghist, int pa, int slot_a, int pb, int slot_b, int slot_c,
                            const uint32_t *run_if) {
    griddep();
    __shared__ uint32_t s[256];
    if (run_if && *run_if == 0u) return;
    const int k = blockIdx.x;
    const int slot = k < pa ? slot_a + k : k < pa + pb ? slot_b + (k - pa) : slot_c + (k - pa - pb);
    uint32_t *h = ghist + 256 * slot;
    const int t = threadIdx.x;
    const uint32_t x = h[t];
    s[t] = x;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        const uint32_t y = t >= o ? s[t - o] : 0u;
        __syncthreads();
        s[t] += y;
        __syncthreads();
    }
    h[t] = s[t] - x;
}

__global__ void __launch_bounds__(kThreads) k_onesweep(const uint64_t *__restrict__ kin,
                                                       const uint32_t *__restrict__ iin, uint64_t *__restrict__ kout,
                                                       uint32_t *__restrict__ iout, uint32_t n, int shift,
                                                       const uint32_t *__restrict__ goff, uint32_t *status,
                                                       uint32_t *ticket, uint32_t *err, uint32_t err_bit,
                                                       const uint32_t *run_if) {
    griddep();
    __shared__ uint32_t s_wc[kWarps][256];  // per-warp digit counts, then per-warp offsets
    __shared__ uint32_t s_base[256];        // global position of the tile's first key of each digit
    __shared__ uint32_t s_lstart[256];      // position of each digit's first key within the tile
    __shared__ uint32_t s_wsum[kWarps];
    __shared__ uint64_t s_buf[kTile];       // the tile in digit order: keys, then indices
    __shared__ uint32_t s_tile;
    if (run_if && *run_if == 0u) return;  // a pass that runs only when a device-side flag is set
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) s_tile = atomicAdd(ticket, 1u);
    for (int k = 0; k < kWarps; k++) s_wc[k][t] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kTile + (uint32_t)w * (32 * kItems);
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t key[kItems];
    uint32_t idx[kItems], rank[kItems];
    // ---- load, then rank: warp w owns keys [base, base + 512) in order
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t i = base + r * 32 + lane;
        const bool valid = i < n;
        key[r] = valid ? __ldcs(&kin[i]) : 0ull;
        idx[r] = valid ? __ldcs(&iin[i]) : 0u;
    }
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t i = base + r * 32 + lane;
        const bool valid = i < n;
        const uint32_t d = (uint32_t)((key[r] >> shift) & 255u);
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const uint32_t bb = __ballot_sync(0xffffffffu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bb : ~bb;
        }
        if (!valid) peers = 1u << lane;
        const uint32_t before = valid ? s_wc[w][d] : 0u;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0) s_wc[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // ---- per digit (thread t = digit): offsets of each warp, tile total
    uint32_t total = 0;
#pragma unroll
    for (int k = 0; k < kWarps; k++) {
        const uint32_t c = s_wc[k][t];
        s_wc[k][t] = total;
        total += c;
    }
    // ---- tile-local start of each digit (exclusive scan of the 256 totals)
    {
        uint32_t x = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[w] = x;
        __syncthreads();
        uint32_t off = 0;
        for (int k = 0; k < w; k++) off += s_wsum[k];
        s_lstart[t] = off + x - total;
    }
    // ---- decoupled look-back over earlier tiles
    uint32_t *st = status + (size_t)tile * 256 + t;
    uint32_t excl = 0;
    if (tile == 0) {
        atomicExch(st, kFlagInc | total);
    } else {
        atomicExch(st, kFlagAgg | total);
        // read up to 8 predecessors per round trip, newest first
        const volatile uint32_t *vs = status;
        int64_t p = (int64_t)tile - 1;
        uint32_t spins = 0;
        bool done = false;
        while (!done) {
            uint32_t v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = p - k >= 0 ? vs[(size_t)(p - k) * 256 + t] : kFlagInc;
            int used = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if (done || used < k) continue;  // stop at the first entry not yet published
                const uint32_t flag = v[k] & ~kValue;
                if (flag == 0u) continue;
                excl += v[k] & kValue;
                used = k + 1;
                if (flag == kFlagInc) done = true;
            }
            p -= used;
            if (!done && used == 0 && ++spins > kSpinLimit) {
                atomicOr(err, err_bit);
                break;
            }
        }
        __threadfence();
        atomicExch(st, kFlagInc | (excl + total));
    }
    s_base[t] = goff[t] + excl;
    __syncthreads();
    // ---- scatter through shared memory: the tile is laid out in digit order,
    // then consecutive threads write consecutive positions of each digit's run
    const uint32_t tcount = min(kTile, n - tile * kTile);
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t i = base + r * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)((key[r] >> shift) & 255u);
            s_buf[s_lstart[d] + s_wc[w][d] + rank[r]] = key[r];
        }
    }
    __syncthreads();
    uint32_t dslot[kItems];
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t q = (uint32_t)t + r * kThreads;
        dslot[r] = 0;
        if (q < tcount) {
            const uint64_t k = s_buf[q];
            const uint32_t d = (uint32_t)((k >> shift) & 255u);
            dslot[r] = d;
            kout[s_base[d] + (q - s_lstart[d])] = k;
        }
    }
    __syncthreads();
    uint32_t *s_idx = reinterpret_cast<uint32_t *>(s_buf);
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t i = base + r * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)((key[r] >> shift) & 255u);
            s_idx[s_lstart[d] + s_wc[w][d] + rank[r]] = idx[r];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; r++) {
        const uint32_t q = (uint32_t)t + r * kThreads;
        if (q < tcount) iout[s_base[dslot[r]] + (q - s_lstart[dslot[r]])] = s_idx[q];
    }
}

}  // namespace

// Scratch: the digit offsets of every slot, then the tile status words of
// every slot, then one ticket per slot.
size_t sort_scratch_bytes(uint32_t n) {
    const size_t tiles = (n + kTile - 1) / kTile;
    return 4 * (kSortSlots * 256 + kSortSlots * tiles * 256 + 64);
}

cudaError_t sort_reset(uint32_t *scratch, uint32_t n, cudaStream_t st) {
    const size_t words = sort_scratch_bytes(n) / 4;
    const unsigned blocks = (unsigned)std::min<size_t>(1184, (words / 4 + 255) / 256);
    return launch_pdl(k_zero_words, dim3(blocks ? blocks : 1), dim3(256), 0, st, scratch, words);
}

cudaError_t sort_histograms(const uint64_t *wa, int pa, int slot_a, const uint64_t *wb, int pb, int slot_b,
                            const uint32_t *wc, int slot_c, uint32_t n, uint32_t *scratch, const uint32_t *run_if,
                            cudaStream_t st, unsigned *launches) {
    if (!wa) pa = 0;
    if (!wb) pb = 0;
    const int np = pa + pb + (wc ? 2 : 0);
    if (np == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<size_t>(1184, (n + 255) / 256);
    launch_pdl(k_hist, dim3(blocks ? blocks : 1), dim3(256), 0, st, wa, pa, slot_a, wb, pb, slot_b, wc, slot_c, n, scratch, run_if);
    launch_pdl(k_hist_scan, dim3(np), dim3(256), 0, st, scratch, pa, slot_a, pb, slot_b, slot_c, run_if);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t sort_pass(const uint64_t *kin, const uint32_t *iin, uint64_t *kout, uint32_t *iout, uint32_t n, int slot,
                      int shift, uint32_t *scratch, uint32_t *err, uint32_t err_bit, const uint32_t *run_if,
                      cudaStream_t st, unsigned *launches) {
    const size_t tiles = (n + kTile - 1) / kTile;
    uint32_t *goff = scratch + 256 * slot;
    uint32_t *status = scratch + kSortSlots * 256 + (size_t)slot * tiles * 256;
    uint32_t *ticket = scratch + kSortSlots * 256 + kSortSlots * tiles * 256 + slot;
    launch_pdl(k_onesweep, dim3((unsigned)tiles), dim3(kThreads), 0, st, kin, iin, kout, iout, n, shift, goff, status, ticket, err,
                                                     err_bit, run_if);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace nbody
