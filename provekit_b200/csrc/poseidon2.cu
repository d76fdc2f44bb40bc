// poseidon2.cu -- BN254 Poseidon2, t = 4, rf = 8, rp = 56, on the device:
//   pkg_poseidon2_permutation_many  poseidon2_permutation (poseidon2/src/permutation.rs:134-177)
//   pkg_poseidon2_hash_many         poseidon2_hash (poseidon2/src/hash.rs:17-47)
// One thread per permutation; state and constants in Montgomery form.  The
// constant tables come from the reference's poseidon2/src/constants.rs via
// gen_poseidon2_constants.py and are copied to __constant__ memory once per
// device.
#include <cstring>
#include <mutex>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "pk_common.cuh"
#include "poseidon2_t4_constants.h"

namespace pk {

__constant__ uint64_t kP2Rc[64][4][4];
__constant__ uint64_t kP2Diag[4][4];

static std::mutex g_p2_mu;
static std::vector<char> g_p2_ready;

static int p2_upload() {
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_p2_mu);
  if ((int)g_p2_ready.size() <= dev) g_p2_ready.resize(dev + 1, 0);
  if (!g_p2_ready[dev]) {
    PK_CUDA(cudaMemcpyToSymbol(kP2Rc, POSEIDON2_T4_RC_MONT, sizeof kP2Rc));
    PK_CUDA(cudaMemcpyToSymbol(kP2Diag, POSEIDON2_T4_DIAG_MONT, sizeof kP2Diag));
    g_p2_ready[dev] = 1;
  }
  return PKG_OK;
}

__device__ __forceinline__ Fr p2_const(const uint64_t* c) {
  Fr r;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    r.v[2 * i] = (uint32_t)c[i];
    r.v[2 * i + 1] = (uint32_t)(c[i] >> 32);
  }
  return r;
}

__device__ __forceinline__ Fr p2_sbox(const Fr& x) {  // x^5
  Fr s = fr_sqr_f64(x);
  s = fr_sqr_f64(s);
  return fr_mul_f64(s, x);
}

// matrix_multiplication_4x4 (permutation.rs:101-120)
__device__ __forceinline__ void p2_ext(Fr (&s)[4]) {
  Fr t0 = fr_add(s[0], s[1]);
  Fr t1 = fr_add(s[2], s[3]);
  Fr t2 = fr_add(fr_add(s[1], s[1]), t1);
  Fr t3 = fr_add(fr_add(s[3], s[3]), t0);
  Fr t4 = fr_add(t1, t1);
  t4 = fr_add(fr_add(t4, t4), t3);
  Fr t5 = fr_add(t0, t0);
  t5 = fr_add(fr_add(t5, t5), t2);
  Fr t6 = fr_add(t3, t5);
  Fr t7 = fr_add(t2, t4);
  s[0] = t6;
  s[1] = t5;
  s[2] = t7;
  s[3] = t4;
}

// internal_m_multiplication (permutation.rs:122-127)
__device__ __forceinline__ void p2_int(Fr (&s)[4]) {
  Fr sum = fr_add(fr_add(s[0], s[1]), fr_add(s[2], s[3]));
#pragma unroll
  for (int i = 0; i < 4; i++) s[i] = fr_add(fr_mul_f64(s[i], p2_const(kP2Diag[i])), sum);
}

__device__ __forceinline__ void p2_permute(Fr (&s)[4]) {
  p2_ext(s);
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = p2_sbox(fr_add(s[i], p2_const(kP2Rc[r][i])));
    p2_ext(s);
  }
#pragma unroll 1
  for (int r = 4; r < 60; r++) {
    s[0] = p2_sbox(fr_add(s[0], p2_const(kP2Rc[r][0])));
    p2_int(s);
  }
#pragma unroll 1
  for (int r = 60; r < 64; r++) {
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = p2_sbox(fr_add(s[i], p2_const(kP2Rc[r][i])));
    p2_ext(s);
  }
}

__global__ void p2_permutation_kernel(uint64_t* __restrict__ states, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr s[4];
#pragma unroll
    for (int k = 0; k < 4; k++) s[k] = fr_load(states, 4 * i + k);
    p2_permute(s);
#pragma unroll
    for (int k = 0; k < 4; k++) fr_store(states, 4 * i + k, s[k]);
  }
}

// Sponge of poseidon2_hash (hash.rs:17-47): rate 3, state[3] = len * 2^64.
__global__ void p2_hash_kernel(const uint64_t* __restrict__ in, size_t len, size_t n, Fr iv,
                               uint64_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr s[4] = {fr_zero(), fr_zero(), fr_zero(), iv};
    Fr cache[3] = {fr_zero(), fr_zero(), fr_zero()};
    int cs = 0;
    for (size_t k = 0; k < len; k++) {
      if (cs == 3) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
          s[j] = fr_add(s[j], cache[j]);
          cache[j] = fr_zero();
        }
        cs = 0;
        p2_permute(s);
      }
      Fr x = fr_load_ro(in, i * len + k);
      if (cs == 0) cache[0] = x;
      else if (cs == 1) cache[1] = x;
      else cache[2] = x;
      cs++;
    }
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (j < cs) s[j] = fr_add(s[j], cache[j]);
    p2_permute(s);
    fr_store(out, i, s[0]);
  }
}

static int p2_grid(size_t n) {
  size_t b = (n + 127) / 128;
  return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sm_count() * 32));
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_poseidon2_permutation_many(uint64_t* states, size_t n, pkg_stream_t stream) {
  if (n == 0) return PKG_OK;
  PK_REQUIRE(states && aligned16(states), "states must be a 16-byte aligned device pointer");
  int rc = p2_upload();
  if (rc) return rc;
  p2_permutation_kernel<<<p2_grid(n), 128, 0, as_stream(stream)>>>(states, n);
  PK_CHECK_LAUNCH("p2_permutation_kernel");
  return PKG_OK;
}

extern "C" int pkg_poseidon2_hash_many(const uint64_t* inputs, size_t len, size_t n, uint64_t* out,
                                       pkg_stream_t stream) {
  if (n == 0) return PKG_OK;
  PK_REQUIRE(out && aligned16(out) && (len == 0 || (inputs && aligned16(inputs))),
             "null or unaligned device pointer");
  int rc = p2_upload();
  if (rc) return rc;
  HostFr iv = HostFr::mul(HostFr::from_u64(len), HostFr::to_mont(HostFr::from_limbs(
                                                        std::vector<uint64_t>{0, 1, 0, 0}.data())));
  Fr ivd;
  memcpy(ivd.v, iv.l, 32);
  p2_hash_kernel<<<p2_grid(n), 128, 0, as_stream(stream)>>>(inputs, len, n, ivd, out);
  PK_CHECK_LAUNCH("p2_hash_kernel");
  return PKG_OK;
}
