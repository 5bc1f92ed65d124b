// Onesweep-style LSD radix sort of (u64 key, u32 index) pairs (sort.cu).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

namespace nbody {

// Histogram and status slots of one sort scratch. A slot holds the digit
// offsets of one pass and that pass's tile status words and ticket; every pass
// of one build takes a different slot.
constexpr int kSortSlots = 34;

// Right shift of pass q (0-based, least significant digit first) when `passes`
// 8-bit digits sort a 63-bit key word from its top bit down: all 64 bits,
// byte-aligned, for 8 passes; otherwise bits [63 - 8 passes, 63), the word's
// top 8 passes key bits (bit 63 is always zero).
__host__ __device__ inline int digit_shift(int passes, int q) { return passes >= 8 ? 8 * q : 63 - 8 * passes + 8 * q; }

// Bytes of device scratch for sorting n pairs (histograms, tile status, tickets).
size_t sort_scratch_bytes(uint32_t n);

// Zeroes the whole scratch (every slot), once per sort.
cudaError_t sort_reset(uint32_t *scratch, uint32_t n, cudaStream_t st);

// Global digit offsets of up to two 63-bit words and a 16-bit word: pa passes
// of wa into slots slot_a.., pb passes of wb into slot_b.., and (wc non-null)
// the two bytes of wc into slots slot_c, slot_c + 1. A word with 0 passes (or
// null) is skipped. The words are given in any order of the same n elements.
// With run_if non-null, nothing happens unless *run_if is non-zero.
cudaError_t sort_histograms(const uint64_t *wa, int pa, int slot_a, const uint64_t *wb, int pb, int slot_b,
                            const uint32_t *wc, int slot_c, uint32_t n, uint32_t *scratch, const uint32_t *run_if,
                            cudaStream_t st, unsigned *launches);

// One stable pass by the 8-bit digit (key >> shift) & 255, with the digit
// offsets, status words and ticket of `slot` (the histogram of that slot must
// have been computed with the same shift). With run_if non-null the pass does
// nothing unless *run_if is non-zero when it starts. A look-back that gives up
// waiting ORs err_bit into *err.
cudaError_t sort_pass(const uint64_t *kin, const uint32_t *iin, uint64_t *kout, uint32_t *iout, uint32_t n, int slot,
                      int shift, uint32_t *scratch, uint32_t *err, uint32_t err_bit, const uint32_t *run_if,
                      cudaStream_t st, unsigned *launches);

}  // namespace nbody
