// Onesweep-style LSD radix sort of (u64 key, u32 index) pairs (sort.cu).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

namespace nbody {

// Bytes of device scratch for sorting n pairs (histograms, tile status, tickets).
size_t sort_scratch_bytes(uint32_t n);

// Zeroes the scratch and computes the global digit offsets of every pass:
// passes 0-7 sort by the bytes of w0, 8-15 of w1, 16-17 of the 16-bit w2
// (npass 16 or 18). The words are given in any order of the same n elements.
cudaError_t sort_prepare(const uint64_t *w0, const uint64_t *w1, const uint32_t *w2, uint32_t n, int npass,
                         uint32_t *scratch, cudaStream_t st, unsigned *launches);

// One stable pass by byte `shift / 8` of the keys, with the digit offsets of
// histogram pass `pass` (0..17) and status words and ticket of its own `slot`
// (0..25; every pass of one sort takes a different slot). With run_if non-null
// the pass does nothing unless *run_if is non-zero when it starts.
// A look-back that gives up waiting ORs err_bit into *err.
cudaError_t sort_pass(const uint64_t *kin, const uint32_t *iin, uint64_t *kout, uint32_t *iout, uint32_t n, int pass,
                      int slot, int shift, uint32_t *scratch, uint32_t *err, uint32_t err_bit, const uint32_t *run_if,
                      cudaStream_t st, unsigned *launches);

}  // namespace nbody
