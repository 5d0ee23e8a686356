// Argsort of 64-bit keys on the GPU (ff_sort.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ffb {

// up to this many keys (with end_bit + 14 < 64) are sorted by one block
// (128 KB of shared memory)
constexpr uint32_t SORT_SMALL = 16384;

// Temporary device bytes argsort_u64 needs for n keys (none on the one-block
// path, which the caller need not know: the figure covers both).
size_t argsort_temp_bytes(uint32_t n);

// keys_out = keys[0, n) in ascending order, pos_out = the input position of
// each; equal keys keep their input order.  Keys are below 2^end_bit.
// keys_out / pos_out must not overlap keys.  *launches (may be null) is
// increased by the number of kernel launches issued.  pdl: the one-block
// sort is launched as a programmatic dependent of the stream's previous
// kernel (which must be a kernel).
cudaError_t argsort_u64(const uint64_t *keys, uint32_t n, int end_bit, uint64_t *keys_out, uint32_t *pos_out,
                        void *tmp, size_t tmp_bytes, cudaStream_t s, unsigned *launches, bool pdl = false);

cudaError_t prewarm_sort_kernels();

}  // namespace ffb
