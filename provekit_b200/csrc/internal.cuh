// internal.cuh -- device-side entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pk {

int merkle_tree_fr_device(const uint64_t* cw, size_t fr_per_leaf, size_t num_leaves, int encoding,
                          uint8_t* layers, cudaStream_t s);
int spmv_device(const uint64_t* row_ptr, const uint32_t* cols, const uint64_t* vals,
                size_t num_rows, size_t num_cols, const uint64_t* x, uint64_t* y, uint32_t* err,
                cudaStream_t s);
int eq_hypercube_device(const uint64_t* r_host, size_t nr, size_t num_entries, uint64_t* out,
                        cudaStream_t s);
// Skyscraper PoW on stream s (synchronous): generic::solve's answer.
int pow_solve_device(const uint64_t challenge[4], const uint64_t threshold[4], cudaStream_t s,
                     uint64_t* nonce_out);
int dot_device(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* d_out, uint64_t* part,
               cudaStream_t s);

}  // namespace pk
