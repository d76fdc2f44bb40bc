// whir.cu -- the data-parallel pieces of WHIR's prove rounds on the device.
//
// The WHIR prover itself lives in the un-vendored `whir` crate (called from
// provekit/prover/src/whir_r1cs.rs:295-301, 378-414).  Its rounds are built
// from the operations below; their arithmetic follows the reference's WHIR
// verifier restated in Go (recursive-verifier/app/utilities/utilities.go,
// recursive-verifier/app/circuit/whir_utilities.go):
//   pkg_whir_fold_coeffs     fold 2^k interleaved messages with the folding
//                            randomness (MultivarPoly weights, utilities.go:16-23)
//   pkg_whir_fold_rows       computeFold over codeword rows (whir_utilities.go:182-188)
//   pkg_poly_eval_many       UnivarPoly at OOD points (utilities.go:25-39)
//   pkg_merkle_open          authentication paths as verifyMerkleTreeProofs
//   pkg_gather_rows          reads them (whir_utilities.go:14-47)
//   pkg_whir_sumcheck_round  one round of the weighted sumcheck, sent as
//                            evaluations at 0, 1, 2 (utilities.go:149-171)
//   pkg_eq_accumulate        w += sum_j c_j eq(p_j, .) for new constraints
//   pkg_stir_indices         getStirChallenges (whir_utilities.go:49-79), host
#include <algorithm>
#include <cstring>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "fr_lazy.cuh"
#include "internal.cuh"
#include "pk_common.cuh"
#include "reduce.cuh"

namespace pk {

constexpr int kMaxFoldK = 6;

// Montgomery field elements passed by value as kernel parameters.
template <int N>
struct FrParams {
  uint32_t v[N][8];
};

template <int N>
__device__ __forceinline__ Fr param_fr(const FrParams<N>& p, int j) {
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = p.v[j][i];
  return r;
}

template <int N>
static void put_param(FrParams<N>& p, int j, const HostFr& x) {
  memcpy(p.v[j], x.l, 32);
}

// w_j = prod_t alpha[t]^(bit t of j): MultivarPoly's coefficient of row entry j.
static void fold_weights(const uint64_t* alpha, unsigned k, FrParams<1 << kMaxFoldK>& W) {
  std::vector<HostFr> w((size_t)1 << k);
  w[0] = HostFr::one();
  for (unsigned t = 0; t < k; t++) {
    const HostFr a = HostFr::from_limbs(alpha + 4 * t);
    const size_t half = size_t(1) << t;
    for (size_t j = 0; j < half; j++) w[j + half] = HostFr::mul(w[j], a);
  }
  for (size_t j = 0; j < w.size(); j++) put_param(W, (int)j, w[j]);
}

// out[i] = sum_j w_j c[j L + i]  (w_0 = 1)
__global__ void whir_fold_coeffs_kernel(const uint64_t* __restrict__ c, size_t L, int m,
                                        const __grid_constant__ FrParams<1 << kMaxFoldK> W,
                                        uint64_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < L;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_load_ro(c, i);
    for (int j = 1; j < m; j++) acc = fr_add(acc, fr_mul_f64(param_fr(W, j), fr_load_ro(c, j * L + i)));
    fr_store(out, i, acc);
  }
}

// out[i] = sum_j w_j rows[i m + j]
__global__ void whir_fold_rows_kernel(const uint64_t* __restrict__ rows, size_t nrows, int m,
                                      const __grid_constant__ FrParams<1 << kMaxFoldK> W,
                                      uint64_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nrows;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_load_ro(rows, i * m);
    for (int j = 1; j < m; j++)
      acc = fr_add(acc, fr_mul_f64(param_fr(W, j), fr_load_ro(rows, i * m + j)));
    fr_store(out, i, acc);
  }
}

// CTA b owns the C coefficients [bC, (b + 1)C) (C a multiple of the CTA
// size); its thread j takes bC + j + 256k for k = 0, 1, ..: Horner in
// y = z^256 from the top.  A power tree in shared memory combines the 256
// thread values, level l joining neighbours 2^l apart with z^(2^l), to
// sum_j acc_j z^j; thread 0 scales it by z^(bC) (from the squares
// z^(C 2^b)), and the CTA values are summed.  Per coefficient one product,
// per thread one more: a per-thread z^t would cost up to log2(threads)
// products per thread, more than the coefficients at mid sizes.
// P.v[0] = z^256, P.v[1 + l] = z^(2^l) (l < 8), P.v[9 + b] = z^(C 2^b).
constexpr int kEvalTreeLevels = 8;  // kRedThreads = 2^8
constexpr int kEvalScaleBits = 10;  // CTAs < 2^10
static_assert(kRedThreads == 1 << kEvalTreeLevels, "one tree level per thread-index bit");

__global__ void __launch_bounds__(kRedThreads) poly_eval_kernel(
    const uint64_t* __restrict__ c, size_t n, size_t C,
    const __grid_constant__ FrParams<1 + kEvalTreeLevels + kEvalScaleBits> P, const RedOut ro) {
  __shared__ Fr tree[kRedThreads];
  const unsigned j = threadIdx.x;
  const size_t c0 = blockIdx.x * C;
  Fr acc = fr_zero();
  if (c0 + j < n) {
    const Fr y = param_fr(P, 0);
    const size_t end = n < c0 + C ? n : c0 + C;
    for (size_t k = (end - 1 - c0 - j) / kRedThreads + 1; k-- > 0;)
      acc = fr_add(fr_mul_f64(acc, y), fr_load_ro(c, c0 + j + (size_t)kRedThreads * k));
  }
  Fr scale = fr_one_mont();
  if (j == 0)
    for (int b = 0; b < kEvalScaleBits; b++)
      if ((blockIdx.x >> b) & 1) scale = fr_mul_f64(scale, param_fr(P, 1 + kEvalTreeLevels + b));
  tree[j] = acc;
  __syncthreads();
#pragma unroll 1
  for (int l = 0; l < kEvalTreeLevels; l++) {
    const unsigned half = kRedThreads >> (l + 1);
    Fr v;
    if (j < half) v = fr_add(tree[2 * j], fr_mul_f64(param_fr(P, 1 + l), tree[2 * j + 1]));
    __syncthreads();
    if (j < half) tree[j] = v;
    __syncthreads();
  }
  Fr out[1] = {fr_zero()};
  if (j == 0) out[0] = fr_mul_f64(tree[0], scale);
  block_finish<1>(out, ro);
}

// path[q depth + l] = node (idx[q] >> l) ^ 1 of level l
__global__ void merkle_open_kernel(const uint8_t* __restrict__ layers, size_t num_leaves,
                                   int depth, const uint64_t* __restrict__ idx, size_t nq,
                                   uint8_t* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq * (size_t)depth;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t q = t / depth;
    const int l = (int)(t % depth);
    size_t off = 0, width = num_leaves;
    for (int j = 0; j < l; j++) {
      off += width;
      width >>= 1;
    }
    const uint4* src = reinterpret_cast<const uint4*>(layers + 32 * (off + ((idx[q] >> l) ^ 1)));
    uint4* dst = reinterpret_cast<uint4*>(out + 32 * t);
    dst[0] = src[0];
    dst[1] = src[1];
  }
}

// rows_out[q][e] = codeword[idx[q]][e]
__global__ void gather_rows_kernel(const uint64_t* __restrict__ cw, size_t row_fr,
                                   const uint64_t* __restrict__ idx, size_t nq,
                                   uint64_t* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq * row_fr;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t q = t / row_fr, e = t % row_fr;
    fr_store(out, t, fr_load_ro(cw, idx[q] * row_fr + e));
  }
}

// One WHIR sumcheck round over f, w (quarter layout when folding, as the
// Spartan rounds): pairs (i, i + q); sums f0 w0, f1 w1, (2f1-f0)(2w1-w0).
// The round kernel's seven products go through one out-of-line call, and the
// kernel is bounded to two CTAs per SM (128 registers): with them inlined the
// folding kernel took 172 registers, one CTA of 256 threads per SM.
static __device__ __noinline__ Fr whir_mul(const Fr a, const Fr b) { return fr_mul_f64(a, b); }

template <bool kFold>
__global__ void __launch_bounds__(kRedThreads, 2) whir_round_kernel(
    uint64_t* __restrict__ f, uint64_t* __restrict__ w, size_t q,
    const __grid_constant__ FrParams<1> A, const RedOut ro) {
  Fr acc[3] = {fr_zero(), fr_zero(), fr_zero()};
  const Fr alpha = param_fr(A, 0);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < q;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr f0 = fr_load(f, i), f1 = fr_load(f, i + q), w0 = fr_load(w, i), w1 = fr_load(w, i + q);
    if (kFold) {
      f0 = fr_add(f0, whir_mul(alpha, fr_sub(fr_load(f, i + 2 * q), f0)));
      f1 = fr_add(f1, whir_mul(alpha, fr_sub(fr_load(f, i + 3 * q), f1)));
      w0 = fr_add(w0, whir_mul(alpha, fr_sub(fr_load(w, i + 2 * q), w0)));
      w1 = fr_add(w1, whir_mul(alpha, fr_sub(fr_load(w, i + 3 * q), w1)));
      fr_store(f, i, f0);
      fr_store(f, i + q, f1);
      fr_store(w, i, w0);
      fr_store(w, i + q, w1);
    }
    acc[0] = fr_add(acc[0], whir_mul(f0, w0));
    acc[1] = fr_add(acc[1], whir_mul(f1, w1));
    const Fr f2 = fr_sub(fr_add(f1, f1), f0), w2 = fr_sub(fr_add(w1, w1), w0);
    acc[2] = fr_add(acc[2], whir_mul(f2, w2));
  }
  block_finish<3>(acc, ro);
}

// tables[j][x] = scale_j * prod_i (bit i of x, top first ? p_j[i] : 1 - p_j[i])
// over k variables; p_j = pts + 4 (j * stride + first).
__global__ void eq_tables_kernel(const uint64_t* __restrict__ pts, size_t stride, size_t first,
                                 int k, const uint64_t* __restrict__ scale, size_t npts,
                                 uint64_t* __restrict__ tables) {
  const size_t per = size_t(1) << k;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < npts * per;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t j = t / per, x = t % per;
    Fr acc = scale ? fr_load_ro(scale, j) : fr_one_mont();
    for (int i = 0; i < k; i++) {
      const Fr p = fr_load_ro(pts, j * stride + first + i);
      const bool bit = (x >> (k - 1 - i)) & 1;
      acc = fr_mul_f64(acc, bit ? p : fr_sub(fr_one_mont(), p));
    }
    fr_store(tables, t, acc);
  }
}

// out[j nv + nv - 1 - i] = z_j^(2^i): the expansion of each univariate point
// into nv coordinates, the top variable first (ExpandFromUnivariate,
// recursive-verifier/app/utilities/utilities.go:183-191).
__global__ void expand_points_kernel(const uint64_t* __restrict__ raw, size_t npts, size_t nv,
                                     uint64_t* __restrict__ out) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < npts;
       j += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_load_ro(raw, j);
    for (size_t i = 0; i < nv; i++) {
      fr_store(out, j * nv + nv - 1 - i, acc);
      acc = fr_sqr_f64(acc);
    }
  }
}

// w[b] += sum_j hi_j[b >> nlo] lo_j[b & (2^nlo - 1)]
__global__ void eq_accumulate_kernel(uint64_t* __restrict__ w, size_t n, int nlo,
                                     const uint64_t* __restrict__ hi, size_t nhi_entries,
                                     const uint64_t* __restrict__ lo, size_t npts) {
  const size_t nlo_entries = size_t(1) << nlo;
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < n;
       b += (size_t)gridDim.x * blockDim.x) {
    // two independent products per step, one on the FP64 pipe and one on
    // the integer pipe (the CIOS routine; the same integers), which issue
    // side by side
    const size_t bh = b >> nlo, bl = b & (nlo_entries - 1);
    Fr acc = fr_load(w, b), acc2 = fr_zero();
    size_t j = 0;
    for (; j + 1 < npts; j += 2) {
      acc = fr_add(acc, fr_mul_f64(fr_load_ro(hi, j * nhi_entries + bh),
                                   fr_load_ro(lo, j * nlo_entries + bl)));
      acc2 = fr_add(acc2, fr_mul(fr_load_ro(hi, (j + 1) * nhi_entries + bh),
                                 fr_load_ro(lo, (j + 1) * nlo_entries + bl)));
    }
    if (j < npts)
      acc = fr_add(acc, fr_mul_f64(fr_load_ro(hi, j * nhi_entries + bh),
                                   fr_load_ro(lo, j * nlo_entries + bl)));
    fr_store(w, b, fr_add(acc, acc2));
  }
}

// The same sum with the products accumulated unreduced (fr_lazy.cuh) and
// reduced once per chunk of lazy::kMaxTerms points: the hi tables carry the
// coefficients times 2^8, which the lazy reduction's 2^-264 takes back to
// a Montgomery product's 2^-256.
__global__ void __launch_bounds__(128, 4) eq_accumulate_lazy_kernel(
    uint64_t* __restrict__ w, size_t n, int nlo, const uint64_t* __restrict__ hi,
    size_t nhi_entries, const uint64_t* __restrict__ lo, size_t npts) {
  const size_t nlo_entries = size_t(1) << nlo;
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < n;
       b += (size_t)gridDim.x * blockDim.x) {
    const size_t bh = b >> nlo, bl = b & (nlo_entries - 1);
    Fr sum = fr_load(w, b);
    for (size_t j0 = 0; j0 < npts; j0 += lazy::kMaxTerms) {
      const size_t j1 = npts - j0 < (size_t)lazy::kMaxTerms ? npts : j0 + lazy::kMaxTerms;
      lazy::Acc acc;
      acc.zero();
#pragma unroll 1
      for (size_t j = j0; j < j1; j++) {
        acc.mac(fr_load_ro(hi, j * nhi_entries + bh), fr_load_ro(lo, j * nlo_entries + bl));
        if ((j - j0) % lazy::kCarryEvery == lazy::kCarryEvery - 1) acc.carry();
      }
      sum = fr_add(sum, acc.finish());
    }
    fr_store(w, b, sum);
  }
}

// Points at and above which the lazy sum is cheaper than a product per term
// (its one reduction per entry costs about a product).
constexpr size_t kLazyEqMinPoints = 4;

}  // namespace pk

using namespace pk;

extern "C" int pkg_whir_fold_coeffs(const uint64_t* coeffs, size_t n, unsigned k,
                                    const uint64_t* alpha, uint64_t* out, pkg_stream_t stream) {
  PK_REQUIRE(k <= (unsigned)kMaxFoldK, "folding factor %u above %d", k, kMaxFoldK);
  PK_REQUIRE(is_pow2(n) && n >= (size_t(1) << k), "length %zu is not a power of two >= 2^%u", n, k);
  PK_REQUIRE(coeffs && out && (k == 0 || alpha), "null pointer");
  PK_REQUIRE(aligned16(coeffs) && aligned16(out), "device buffers must be 16-byte aligned");
  FrParams<1 << kMaxFoldK> W;
  memset(&W, 0, sizeof W);
  fold_weights(alpha, k, W);
  const size_t L = n >> k;
  whir_fold_coeffs_kernel<<<ew_grid(L), 256, 0, as_stream(stream)>>>(coeffs, L, 1 << k, W, out);
  PK_CHECK_LAUNCH("whir_fold_coeffs_kernel");
  return PKG_OK;
}

extern "C" int pkg_whir_fold_rows(const uint64_t* rows, size_t nrows, unsigned k,
                                  const uint64_t* alpha, uint64_t* out, pkg_stream_t stream) {
  PK_REQUIRE(k <= (unsigned)kMaxFoldK, "folding factor %u above %d", k, kMaxFoldK);
  if (nrows == 0) return PKG_OK;
  PK_REQUIRE(rows && out && (k == 0 || alpha), "null pointer");
  PK_REQUIRE(aligned16(rows) && aligned16(out), "device buffers must be 16-byte aligned");
  FrParams<1 << kMaxFoldK> W;
  memset(&W, 0, sizeof W);
  fold_weights(alpha, k, W);
  whir_fold_rows_kernel<<<ew_grid(nrows), 256, 0, as_stream(stream)>>>(rows, nrows, 1 << k, W, out);
  PK_CHECK_LAUNCH("whir_fold_rows_kernel");
  return PKG_OK;
}

extern "C" int pkg_poly_eval_many(const uint64_t* coeffs, size_t n, const uint64_t* points,
                                  size_t npts, uint64_t* out, pkg_stream_t stream) {
  if (npts == 0) return PKG_OK;
  PK_REQUIRE(points && out, "null pointer");
  if (n == 0) {
    memset(out, 0, 32 * npts);
    return PKG_OK;
  }
  PK_REQUIRE(coeffs && aligned16(coeffs), "null or unaligned coefficients");
  PK_REQUIRE(n < (size_t(1) << 40), "too many coefficients");
  cudaStream_t s = as_stream(stream);
  // at least kEvalMin coefficients per thread, up to 4 CTAs per SM (and
  // fewer than 2^kEvalScaleBits CTAs); C coefficients per CTA
  constexpr size_t kEvalMin = 4;
  const size_t gmax = std::min<size_t>((size_t)sm_count() * 4, (size_t(1) << kEvalScaleBits) - 1);
  size_t g = std::max<size_t>(1, std::min(gmax, (n + kRedThreads * kEvalMin - 1) /
                                                    (kRedThreads * kEvalMin)));
  const size_t per = (n + kRedThreads * g - 1) / (kRedThreads * g);
  const size_t C = per * kRedThreads;
  g = (n + C - 1) / C;
  // up to kFusedSlotFr points: each launch writes its value to the thread's
  // fused slots; more points: partials, one summing launch per point
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  const bool fused = npts <= kFusedSlotFr;
  Scratch scr;
  if (!fused && (rc = scr.alloc(32 * ((size_t)g + npts), s))) return rc;
  uint64_t* part = fused ? fs.part : static_cast<uint64_t*>(scr.ptr);
  uint64_t* d_out = fused ? fs.dev : part + 4 * (size_t)g;
  for (size_t j = 0; j < npts; j++) {
    const HostFr z = HostFr::from_limbs(points + 4 * j);
    FrParams<1 + kEvalTreeLevels + kEvalScaleBits> P;
    HostFr sq = z;
    for (int l = 0; l < kEvalTreeLevels; l++) {  // z^(2^l), then z^256
      put_param(P, 1 + l, sq);
      sq = HostFr::mul(sq, sq);
    }
    put_param(P, 0, sq);
    sq = HostFr::pow_u64(z, C);
    for (int b = 0; b < kEvalScaleBits; b++) {  // z^(C 2^b)
      put_param(P, 1 + kEvalTreeLevels + b, sq);
      sq = HostFr::mul(sq, sq);
    }
    const RedOut ro = {part, fused ? fs.ticket : nullptr, fused ? d_out + 4 * j : nullptr,
                       fused ? fused_next_seq() : 0u};
    poly_eval_kernel<<<(unsigned)g, kRedThreads, 0, s>>>(coeffs, n, C, P, ro);
    PK_CHECK_LAUNCH("poly_eval_kernel");
    if (!fused) {
      sum_partials_kernel<1><<<1, kRedThreads, 0, s>>>(part, (int)g, d_out + 4 * j);
      PK_CHECK_LAUNCH("sum_partials_kernel");
    }
  }
  return fused ? fused_read(out, fs, 32 * npts, s) : read_small(out, d_out, 32 * npts, s);
}

extern "C" int pkg_merkle_open(const uint8_t* layers, size_t num_leaves, const uint64_t* indices,
                               size_t nq, uint8_t* paths, pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(num_leaves), "num_leaves %zu is not a power of two", num_leaves);
  const int depth = log2_exact(num_leaves);
  if (nq == 0 || depth == 0) return PKG_OK;
  PK_REQUIRE(layers && indices && paths && aligned16(layers), "null or unaligned pointer");
  for (size_t q = 0; q < nq; q++)
    PK_REQUIRE(indices[q] < num_leaves, "index %llu out of range (%zu leaves)",
               (unsigned long long)indices[q], num_leaves);
  cudaStream_t s = as_stream(stream);
  Scratch scr;
  const size_t idx_bytes = (8 * nq + 255) & ~size_t(255);
  int rc = scr.alloc(idx_bytes + 32 * nq * depth, s);
  if (rc) return rc;
  uint64_t* d_idx = static_cast<uint64_t*>(scr.ptr);
  uint8_t* d_out = static_cast<uint8_t*>(scr.ptr) + idx_bytes;
  PK_CUDA(cudaMemcpyAsync(d_idx, indices, 8 * nq, cudaMemcpyHostToDevice, s));
  merkle_open_kernel<<<ew_grid(nq * depth), 256, 0, s>>>(layers, num_leaves, depth, d_idx, nq, d_out);
  PK_CHECK_LAUNCH("merkle_open_kernel");
  PK_CUDA(cudaMemcpyAsync(paths, d_out, 32 * nq * depth, cudaMemcpyDeviceToHost, s));
  PK_CUDA(cudaStreamSynchronize(s));
  return PKG_OK;
}

extern "C" int pkg_gather_rows(const uint64_t* codeword, size_t fr_per_row, size_t num_rows,
                               const uint64_t* indices, size_t nq, uint64_t* rows,
                               pkg_stream_t stream) {
  if (nq == 0 || fr_per_row == 0) return PKG_OK;
  PK_REQUIRE(codeword && indices && rows && aligned16(codeword), "null or unaligned pointer");
  for (size_t q = 0; q < nq; q++)
    PK_REQUIRE(indices[q] < num_rows, "index %llu out of range (%zu rows)",
               (unsigned long long)indices[q], num_rows);
  cudaStream_t s = as_stream(stream);
  Scratch scr;
  const size_t idx_bytes = (8 * nq + 255) & ~size_t(255);
  int rc = scr.alloc(idx_bytes + 32 * nq * fr_per_row, s);
  if (rc) return rc;
  uint64_t* d_idx = static_cast<uint64_t*>(scr.ptr);
  uint64_t* d_out = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(scr.ptr) + idx_bytes);
  PK_CUDA(cudaMemcpyAsync(d_idx, indices, 8 * nq, cudaMemcpyHostToDevice, s));
  gather_rows_kernel<<<ew_grid(nq * fr_per_row), 256, 0, s>>>(codeword, fr_per_row, d_idx, nq, d_out);
  PK_CHECK_LAUNCH("gather_rows_kernel");
  PK_CUDA(cudaMemcpyAsync(rows, d_out, 32 * nq * fr_per_row, cudaMemcpyDeviceToHost, s));
  PK_CUDA(cudaStreamSynchronize(s));
  return PKG_OK;
}

namespace pk {
// pkg_gather_rows + pkg_merkle_open of the same indices with one upload and
// one synchronisation.
int open_rows_device(const uint64_t* codeword, size_t fr_per_row, size_t num_rows,
                     const uint8_t* layers, const uint64_t* indices, size_t nq, uint64_t* rows,
                     uint8_t* paths, cudaStream_t s, bool sync) {
  if (nq == 0) return PKG_OK;
  const int depth = log2_exact(num_rows);
  for (size_t q = 0; q < nq; q++)
    PK_REQUIRE(indices[q] < num_rows, "index %llu out of range (%zu rows)",
               (unsigned long long)indices[q], num_rows);
  Scratch scr;
  const size_t idx_bytes = (8 * nq + 255) & ~size_t(255);
  const size_t row_bytes = (32 * nq * fr_per_row + 255) & ~size_t(255);
  int rc = scr.alloc(idx_bytes + row_bytes + 32 * nq * (size_t)depth + 32, s);
  if (rc) return rc;
  uint64_t* d_idx = static_cast<uint64_t*>(scr.ptr);
  uint64_t* d_rows = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(scr.ptr) + idx_bytes);
  uint8_t* d_paths = static_cast<uint8_t*>(scr.ptr) + idx_bytes + row_bytes;
  PK_CUDA(cudaMemcpyAsync(d_idx, indices, 8 * nq, cudaMemcpyHostToDevice, s));
  gather_rows_kernel<<<ew_grid(nq * fr_per_row), 256, 0, s>>>(codeword, fr_per_row, d_idx, nq,
                                                              d_rows);
  PK_CHECK_LAUNCH("gather_rows_kernel");
  if (depth) {
    merkle_open_kernel<<<ew_grid(nq * depth), 256, 0, s>>>(layers, num_rows, depth, d_idx, nq,
                                                           d_paths);
    PK_CHECK_LAUNCH("merkle_open_kernel");
  }
  if (!sync) {
    PK_CUDA(cudaMemcpyAsync(rows, d_rows, 32 * nq * fr_per_row, cudaMemcpyDeviceToHost, s));
    if (depth)
      PK_CUDA(cudaMemcpyAsync(paths, d_paths, 32 * nq * (size_t)depth, cudaMemcpyDeviceToHost, s));
    return PKG_OK;
  }
  const HostRead reads[2] = {{rows, d_rows, 32 * nq * fr_per_row},
                             {paths, d_paths, depth ? 32 * nq * (size_t)depth : 0}};
  return read_small(reads, depth ? 2 : 1, s);
}
}  // namespace pk

extern "C" int pkg_stir_indices(const uint8_t* bytes, size_t folded_domain_size, size_t nq,
                                uint64_t* out) {
  PK_REQUIRE(is_pow2(folded_domain_size), "folded domain size %zu is not a power of two",
             folded_domain_size);
  if (nq == 0) return PKG_OK;
  PK_REQUIRE(bytes && out, "null pointer");
  const int bits = log2_exact(folded_domain_size);
  const size_t nbytes = (size_t)(bits + 7) / 8;
  for (size_t i = 0; i < nq; i++) {
    uint64_t v = 0;
    for (size_t j = 0; j < nbytes; j++) v = (v << 8) | bytes[i * nbytes + j];
    out[i] = bits >= 64 ? v : (v & ((uint64_t(1) << bits) - 1));
  }
  return PKG_OK;
}

extern "C" int pkg_whir_sumcheck_round(uint64_t* f, uint64_t* w, size_t size, const uint64_t* fold,
                                       uint64_t out[12], pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(size) && size >= 2, "table size %zu must be a power of two >= 2", size);
  PK_REQUIRE(!fold || size >= 4, "folding needs size >= 4 (got %zu)", size);
  PK_REQUIRE(f && w && out && aligned16(f) && aligned16(w), "null or unaligned pointer");
  cudaStream_t s = as_stream(stream);
  const size_t q = fold ? size / 4 : size / 2;
  const int g = red_grid(q);
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  uint64_t* part = fs.part;  // g <= 4 CTAs per SM
  FrParams<1> A;
  memset(&A, 0, sizeof A);
  if (fold) memcpy(A.v[0], fold, 32);
  const RedOut ro = {part, fs.ticket, fs.dev, fused_next_seq()};
  if (fold)
    whir_round_kernel<true><<<g, kRedThreads, 0, s>>>(f, w, q, A, ro);
  else
    whir_round_kernel<false><<<g, kRedThreads, 0, s>>>(f, w, q, A, ro);
  PK_CHECK_LAUNCH("whir_round_kernel");
  return fused_read(out, fs, 96, s);
}

namespace pk {
int eq_accumulate_device(uint64_t* w, size_t nv, const uint64_t* points, const uint64_t* coeffs,
                         size_t npts, cudaStream_t s, bool sync, bool expanded) {
  if (npts == 0) return PKG_OK;
  const int nhi = (int)(nv + 1) / 2, nlo = (int)nv - nhi;
  const size_t nh = size_t(1) << nhi, nl = size_t(1) << nlo, n = size_t(1) << nv;
  Scratch scr;
  const size_t pts_fr = npts * (nv ? nv : 1);
  // [expanded points | coefficients | hi tables | lo tables | raw points]
  int rc = scr.alloc(32 * (pts_fr + npts + npts * (nh + nl) + (expanded ? 0 : npts)), s);
  if (rc) return rc;
  uint64_t* d_pts = static_cast<uint64_t*>(scr.ptr);
  uint64_t* d_cf = d_pts + 4 * pts_fr;
  uint64_t* d_hi = d_cf + 4 * npts;
  uint64_t* d_lo = d_hi + 4 * npts * nh;
  if (nv && expanded) {
    PK_CUDA(cudaMemcpyAsync(d_pts, points, 32 * npts * nv, cudaMemcpyHostToDevice, s));
  } else if (nv) {
    uint64_t* d_raw = d_lo + 4 * npts * nl;
    PK_CUDA(cudaMemcpyAsync(d_raw, points, 32 * npts, cudaMemcpyHostToDevice, s));
    expand_points_kernel<<<ew_grid(npts), 256, 0, s>>>(d_raw, npts, nv, d_pts);
    PK_CHECK_LAUNCH("expand_points_kernel");
  }
  // hi tables carry the coefficient (times 2^8 for the lazy sum), lo tables
  // are plain eq tables
  const bool use_lazy = npts >= kLazyEqMinPoints;
  if (use_lazy) {
    // pageable: staged before cudaMemcpyAsync returns
    std::vector<HostFr> cf8(npts);
    const HostFr m8 = HostFr::from_limbs(lazy::kMont2e8);
    for (size_t j = 0; j < npts; j++) cf8[j] = HostFr::mul(HostFr::from_limbs(coeffs + 4 * j), m8);
    PK_CUDA(cudaMemcpyAsync(d_cf, cf8[0].l, 32 * npts, cudaMemcpyHostToDevice, s));
  } else {
    PK_CUDA(cudaMemcpyAsync(d_cf, coeffs, 32 * npts, cudaMemcpyHostToDevice, s));
  }
  eq_tables_kernel<<<ew_grid(npts * nh), 256, 0, s>>>(d_pts, nv, 0, nhi, d_cf, npts, d_hi);
  PK_CHECK_LAUNCH("eq_tables_kernel");
  eq_tables_kernel<<<ew_grid(npts * nl), 256, 0, s>>>(d_pts, nv, nhi, nlo, nullptr, npts, d_lo);
  PK_CHECK_LAUNCH("eq_tables_kernel");
  if (use_lazy) {
    const int grid = (int)std::max<size_t>(
        1, std::min<size_t>((n + 127) / 128, (size_t)sm_count() * 4 * 8));
    eq_accumulate_lazy_kernel<<<grid, 128, 0, s>>>(w, n, nlo, d_hi, nh, d_lo, npts);
    PK_CHECK_LAUNCH("eq_accumulate_lazy_kernel");
  } else {
    eq_accumulate_kernel<<<ew_grid(n), 256, 0, s>>>(w, n, nlo, d_hi, nh, d_lo, npts);
    PK_CHECK_LAUNCH("eq_accumulate_kernel");
  }
  // host sources in pinned memory must outlive their async copies; pageable
  // ones are staged before cudaMemcpyAsync returns
  if (sync) PK_CUDA(cudaStreamSynchronize(s));
  return PKG_OK;
}
}  // namespace pk

extern "C" int pkg_eq_accumulate(uint64_t* w, size_t nv, const uint64_t* points,
                                 const uint64_t* coeffs, size_t npts, pkg_stream_t stream) {
  PK_REQUIRE(nv < 40, "too many variables (%zu)", nv);
  if (npts == 0) return PKG_OK;
  PK_REQUIRE(w && points && coeffs && aligned16(w), "null or unaligned pointer");
  return eq_accumulate_device(w, nv, points, coeffs, npts, as_stream(stream), true);
}
