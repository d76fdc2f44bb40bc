// ntt_internal.cuh -- NTT entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pk {

// The RS-encode layout as the input of a transform's first pass
// (provekit/common/src/ntt.rs:72-95): element x of each replicated block of
// `chunk` = coset_size * M elements is messages[x % M][x / M] for x < L*M,
// then masks[x - L*M], then zero.
struct NttSource {
  const uint64_t* messages;
  const uint64_t* masks;
  uint64_t M, L, mask_len, chunk;
};

// Ensure the device twiddle table covers `order`; returns its device pointer.
int roots_reserve(size_t order, const uint64_t** out);
// Global stages [t_begin, t_end) of an N-point transform over M interleaved
// columns, in place.  With src, the first pass reads its input from the
// RS-encode layout instead of data (the transpose and coset replication fused
// into its loads).
int ntt_stages(uint64_t* data, size_t N, size_t M, int t_begin, int t_end, const uint64_t* roots,
               cudaStream_t stream, const NttSource* src = nullptr);
int ntt_validate(size_t len, size_t codeword_size, size_t num_groups, int* noop);
int ntt_nr_device(uint64_t* values, size_t len, size_t codeword_size, size_t num_groups,
                  cudaStream_t stream);
int intt_rn_device(uint64_t* values, size_t len, cudaStream_t stream);
// ntt_nr over len elements whose input is the RS-encode layout `src` (out is
// written, never read before the first pass).
int ntt_nr_from_source(uint64_t* out, size_t len, size_t codeword_size, size_t num_groups,
                       const NttSource& src, cudaStream_t stream);

}  // namespace pk
