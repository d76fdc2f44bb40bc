// ntt_internal.cuh -- NTT entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pk {

// Ensure the device twiddle table covers `order`; returns its device pointer.
int roots_reserve(size_t order, const uint64_t** out);
// Global stages [t_begin, t_end) of an N-point transform over M interleaved
// columns, in place.
int ntt_stages(uint64_t* data, size_t N, size_t M, int t_begin, int t_end, const uint64_t* roots,
               cudaStream_t stream);
int ntt_validate(size_t len, size_t codeword_size, size_t num_groups, int* noop);
int ntt_nr_device(uint64_t* values, size_t len, size_t codeword_size, size_t num_groups,
                  cudaStream_t stream);
int intt_rn_device(uint64_t* values, size_t len, cudaStream_t stream);

}  // namespace pk
