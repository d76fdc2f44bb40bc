// Element-wise Fr operations over device arrays on either multiply pipe:
// the FP64-pipe routines (fr_f64.cuh) that the NTT and Skyscraper kernels use,
// and the integer-pipe ones (fr.cuh).  A parity and microbenchmark surface
// for the field arithmetic itself (the reference's scalar_mul / scalar_sqr,
// skyscraper/bn254-multiplier/src/scalar.rs:12-132, and ark-ff's
// from_montgomery).
#include "fr.cuh"
#include "fr_f64.cuh"
#include "pk_common.cuh"

namespace pk {

template <int kOp>
__global__ void fr_op_kernel(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                             uint64_t* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const Fr x = fr_load_ro(a, i);
    Fr r;
    if (kOp == PKG_FR_MUL_F64) r = fr_mul_f64(x, fr_load_ro(b, i));
    if (kOp == PKG_FR_SQR_F64) r = fr_sqr_f64(x);
    if (kOp == PKG_FR_FROM_MONT_F64) r = fr_from_mont_f64(x);
    if (kOp == PKG_FR_MUL_INT) r = fr_mul(x, fr_load_ro(b, i));
    if (kOp == PKG_FR_SQR_INT) r = fr_sqr(x);
    if (kOp == PKG_FR_FROM_MONT_INT) r = fr_from_mont(x);
    fr_store(out, i, r);
  }
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_fr_mul_batch(const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n,
                                int op, pkg_stream_t stream) {
  PK_REQUIRE(op >= PKG_FR_MUL_F64 && op <= PKG_FR_FROM_MONT_INT, "unknown Fr op %d", op);
  if (n == 0) return PKG_OK;
  const bool binary = op == PKG_FR_MUL_F64 || op == PKG_FR_MUL_INT;
  PK_REQUIRE(a && out && (b || !binary), "null pointer");
  PK_REQUIRE(aligned16(a) && aligned16(out) && (!binary || aligned16(b)),
             "device buffers must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  const int threads = 256;
  const size_t want = (n + threads - 1) / threads;
  const int g = (int)(want < 148 * 64 ? want : 148 * 64);
  switch (op) {
    case PKG_FR_MUL_F64: fr_op_kernel<PKG_FR_MUL_F64><<<g, threads, 0, s>>>(a, b, out, n); break;
    case PKG_FR_SQR_F64: fr_op_kernel<PKG_FR_SQR_F64><<<g, threads, 0, s>>>(a, b, out, n); break;
    case PKG_FR_FROM_MONT_F64:
      fr_op_kernel<PKG_FR_FROM_MONT_F64><<<g, threads, 0, s>>>(a, b, out, n);
      break;
    case PKG_FR_MUL_INT: fr_op_kernel<PKG_FR_MUL_INT><<<g, threads, 0, s>>>(a, b, out, n); break;
    case PKG_FR_SQR_INT: fr_op_kernel<PKG_FR_SQR_INT><<<g, threads, 0, s>>>(a, b, out, n); break;
    default: fr_op_kernel<PKG_FR_FROM_MONT_INT><<<g, threads, 0, s>>>(a, b, out, n); break;
  }
  PK_CHECK_LAUNCH("fr_op_kernel");
  return PKG_OK;
}
