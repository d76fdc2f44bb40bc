// rs_internal.cuh -- RS encoder entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pk {

int rs_plan(size_t num_messages, size_t message_length, size_t mask_len, size_t codeword_length,
            size_t* coset_size_out, size_t* num_cosets_out);
int rs_encode_device(const uint64_t* messages, size_t num_messages, size_t message_length,
                     const uint64_t* masks, size_t mask_len, size_t codeword_length,
                     uint64_t* out, cudaStream_t stream);

}  // namespace pk
