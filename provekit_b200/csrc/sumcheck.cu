// sumcheck.cu -- the Spartan side of the prover on the device:
//   pkg_spartan_round      one round of run_zk_sumcheck_prover's map-reduce
//                          (provekit/prover/src/whir_r1cs.rs:551-559 over
//                          sumcheck_fold_map_reduce, provekit/common/src/utils/sumcheck.rs:14-102)
//   pkg_spartan_sumcheck   the whole zk-sumcheck (whir_r1cs.rs:519-621), rounds
//                          on the device, round-polynomial bookkeeping and the
//                          transcript on the host
//   pkg_eq_hypercube       calculate_evaluations_over_boolean_hypercube_for_eq (sumcheck.rs:108-153)
//   pkg_spmv_csr           HydratedSparseMatrix * &[Fr] (sparse_matrix.rs:606-627)
//   pkg_csr_transpose      SparseMatrix::transpose (sparse_matrix.rs:409), as a counting sort
//   pkg_hadamard_pad       c = a o b padded with zeros (calculate_witness_bounds, sumcheck.rs:163-179)
//   pkg_dot                whir::algebra::dot (whir_r1cs.rs:614-617, 637, 650)
//   pkg_transcript_*       host Fiat-Shamir transcript stand-in (see the header)
//
// Reductions use the block-wide sums of reduce.cuh.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "fr_lazy.cuh"
#include "pk_common.cuh"
#include "reduce.cuh"
#include "sky_host.hpp"
#include "sumcheck_device.cuh"

namespace pk {


struct Tables4 {
  uint64_t* t[4];  // a, b, c, eq
};

// kFold: current size s = 4q, folded in place, then pairs (t[j], t[j+q]);
// !kFold: size s = 2q, pairs (t[j], t[j+q]).
template <bool kFold>
__global__ void __launch_bounds__(kRedThreads) spartan_round_kernel(Tables4 tabs, size_t q,
                                                                     Fr fold, const RedOut ro) {
  Fr acc[3] = {fr_zero(), fr_zero(), fr_zero()};
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < q;
       j += (size_t)gridDim.x * blockDim.x)
    spartan_pair<kFold>(tabs.t, j, q, fold, acc);
  block_finish<3>(acc, ro);
}

// eq over a block of variables: out[x] = prod_i (bit_i(x) ? r_i : 1 - r_i)
// with r_0 on the most significant of nr bits.
__global__ void eq_small_kernel(const uint64_t* __restrict__ r, int nr, uint64_t* __restrict__ out) {
  size_t n = size_t(1) << nr;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n;
       x += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_one_mont();
    for (int i = 0; i < nr; i++) {
      Fr ri = fr_load_ro(r, i);
      Fr f = ((x >> (nr - 1 - i)) & 1) ? ri : fr_sub(fr_one_mont(), ri);
      acc = fr_mul_f64(acc, f);
    }
    fr_store(out, x, acc);
  }
}

// out[x] = hi[x >> nlo] * lo[x & (2^nlo - 1)] for x < num_entries.
__global__ void eq_combine_kernel(const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo,
                                  int nlo, size_t num_entries, uint64_t* __restrict__ out) {
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < num_entries;
       x += (size_t)gridDim.x * blockDim.x) {
    fr_store(out, x, fr_mul_f64(fr_load_ro(hi, x >> nlo), fr_load_ro(lo, x & ((size_t(1) << nlo) - 1))));
  }
}

// Column indices >= num_cols are skipped and flagged in *err (the reference
// panics on them); the entry point turns the flag into an error status.
__global__ void spmv_csr_kernel(const uint64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                                const uint64_t* __restrict__ vals, size_t num_rows, size_t num_cols,
                                const uint64_t* __restrict__ x, uint64_t* __restrict__ y,
                                uint32_t* __restrict__ err) {
  for (size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x; row < num_rows;
       row += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_zero();
    for (uint64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) {
      const uint32_t col = cols[k];
      if (col >= num_cols) {
        atomicOr(err, 1u);
        continue;
      }
      acc = fr_add(acc, fr_mul_f64(fr_load_ro(vals, k), fr_load_ro(x, col)));
    }
    fr_store(y, row, acc);
  }
}

// The same product in two balanced passes, for large matrices whose row
// lengths vary (a transposed R1CS matrix: 0 to ~10 entries per witness
// column): one thread per nonzero forms vals[k] * x[cols[k]] into prod[k],
// then one thread per row adds its run of prod -- so a warp's Montgomery
// products no longer wait for its longest row.
__global__ void spmv_products_kernel(const uint32_t* __restrict__ cols,
                                     const uint64_t* __restrict__ vals, size_t nnz,
                                     size_t num_cols, const uint64_t* __restrict__ x,
                                     uint64_t* __restrict__ prod, uint32_t* __restrict__ err) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nnz;
       k += (size_t)gridDim.x * blockDim.x) {
    const uint32_t col = cols[k];
    Fr v = fr_zero();
    if (col >= num_cols)
      atomicOr(err, 1u);
    else
      v = fr_mul_f64(fr_load_ro(vals, k), fr_load_ro(x, col));
    fr_store(prod, k, v);
  }
}

__global__ void spmv_rowsum_kernel(const uint64_t* __restrict__ row_ptr,
                                   const uint64_t* __restrict__ prod, size_t num_rows,
                                   uint64_t* __restrict__ y) {
  for (size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x; row < num_rows;
       row += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_zero();
    for (uint64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) acc = fr_add(acc, fr_load_ro(prod, k));
    fr_store(y, row, acc);
  }
}

// calculate_witness_bounds (sumcheck.rs:163-179) in one pass over the rows:
// a_i = <A_i, w>, b_i = <B_i, w>, c_i = a_i b_i for i < num_rows, and zeros
// up to the padded size (the three tables of the zk-sumcheck).  Column
// indices >= num_cols are skipped and flagged in *err.
__global__ void witness_bounds_kernel(const uint64_t* __restrict__ rpa,
                                      const uint32_t* __restrict__ ca,
                                      const uint64_t* __restrict__ va,
                                      const uint64_t* __restrict__ rpb,
                                      const uint32_t* __restrict__ cb,
                                      const uint64_t* __restrict__ vb, size_t num_rows,
                                      size_t num_cols, size_t padded,
                                      const uint64_t* __restrict__ w, uint64_t* __restrict__ ta,
                                      uint64_t* __restrict__ tb, uint64_t* __restrict__ tc,
                                      uint32_t* __restrict__ err) {
  for (size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x; row < padded;
       row += (size_t)gridDim.x * blockDim.x) {
    Fr a = fr_zero(), b = fr_zero(), c = fr_zero();
    if (row < num_rows) {
      for (uint64_t k = rpa[row]; k < rpa[row + 1]; k++) {
        const uint32_t col = ca[k];
        if (col >= num_cols) {
          atomicOr(err, 1u);
          continue;
        }
        a = fr_add(a, fr_mul_f64(fr_load_ro(va, k), fr_load_ro(w, col)));
      }
      for (uint64_t k = rpb[row]; k < rpb[row + 1]; k++) {
        const uint32_t col = cb[k];
        if (col >= num_cols) {
          atomicOr(err, 1u);
          continue;
        }
        b = fr_add(b, fr_mul_f64(fr_load_ro(vb, k), fr_load_ro(w, col)));
      }
      c = fr_mul_f64(a, b);
    }
    fr_store(ta, row, a);
    fr_store(tb, row, b);
    fr_store(tc, row, c);
  }
}

__global__ void hadamard_pad_kernel(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                                    size_t n, size_t padded, uint64_t* __restrict__ c) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < padded;
       i += (size_t)gridDim.x * blockDim.x)
    fr_store(c, i, i < n ? fr_mul_f64(fr_load_ro(a, i), fr_load_ro(b, i)) : fr_zero());
}

// The products are summed unreduced (fr_lazy.cuh) and reduced once per
// thread; each CTA's sum is then scaled by 2^8 (the lazy reduction divides
// by 2^264 where a Montgomery product divides by 2^256).
__global__ void __launch_bounds__(kRedThreads) dot_kernel(const uint64_t* __restrict__ a,
                                                        const uint64_t* __restrict__ b, size_t n,
                                                        const RedOut ro) {
  Fr acc[1] = {fr_zero()};
  lazy::Acc la;
  la.zero();
  int terms = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    la.mac(fr_load_ro(a, i), fr_load_ro(b, i));
    if (++terms % lazy::kCarryEvery == 0) la.carry();
    if (terms == lazy::kMaxTerms) {
      acc[0] = fr_add(acc[0], la.finish());
      la.zero();
      terms = 0;
    }
  }
  if (terms) acc[0] = fr_add(acc[0], la.finish());
  const Fr s8 = lazy::mont_2e8();
  block_finish<1>(acc, ro, &s8);
}

// ---- CSR transpose: count, exclusive scan, scatter ------------------------
__global__ void csr_count_cols_kernel(const uint32_t* __restrict__ cols, size_t nnz,
                                      size_t num_cols, uint32_t* __restrict__ counts,
                                      uint32_t* __restrict__ err) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nnz;
       k += (size_t)gridDim.x * blockDim.x) {
    if (cols[k] >= num_cols) {
      atomicOr(err, 1u);
      continue;
    }
    atomicAdd(&counts[cols[k]], 1u);
  }
}

__global__ void csr_scatter_kernel(const uint64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                                   const uint64_t* __restrict__ vals, size_t num_rows, size_t num_cols,
                                   unsigned long long* __restrict__ cursor,
                                   uint32_t* __restrict__ cols_t, uint64_t* __restrict__ vals_t) {
  for (size_t row = blockIdx.x * (size_t)blockDim.x + threadIdx.x; row < num_rows;
       row += (size_t)gridDim.x * blockDim.x) {
    for (uint64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) {
      if (cols[k] >= num_cols) continue;  // flagged by csr_count_cols_kernel
      unsigned long long pos = atomicAdd(&cursor[cols[k]], 1ull);
      cols_t[pos] = (uint32_t)row;
      fr_store(vals_t, pos, fr_load_ro(vals, k));
    }
  }
}

__global__ void widen_kernel(const uint32_t* __restrict__ in, size_t n, unsigned long long* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}


// One Spartan round on device tables; the round kernel writes 3 Fr (f0,
// f(-1), f(inf)) to out (the thread's fused slots, whose ticket it takes).
// part: >= red_grid(q) * 3 Fr of scratch.
int spartan_round_device(uint64_t* a, uint64_t* b, uint64_t* c, uint64_t* eq, size_t size,
                         const uint64_t* fold_host, uint64_t* part, uint64_t* out,
                         cudaStream_t s, unsigned* ticket) {
  Tables4 tabs = {{a, b, c, eq}};
  Fr f;
  memset(&f, 0, sizeof f);
  size_t q;
  int g;
  const RedOut ro = {part, ticket, out, ticket ? fused_next_seq() : 0u};
  if (fold_host) {
    memcpy(f.v, fold_host, 32);
    q = size / 4;
    g = red_grid(q);
    spartan_round_kernel<true><<<g, kRedThreads, 0, s>>>(tabs, q, f, ro);
  } else {
    q = size / 2;
    g = red_grid(q);
    spartan_round_kernel<false><<<g, kRedThreads, 0, s>>>(tabs, q, f, ro);
  }
  PK_CHECK_LAUNCH("spartan_round_kernel");
  return PKG_OK;
}

int eq_hypercube_device(const uint64_t* r_host, size_t nr, size_t num_entries, uint64_t* out,
                        cudaStream_t s, bool sync) {
  if (num_entries == 0) return PKG_OK;
  PK_REQUIRE(nr < 40 && num_entries <= (size_t(1) << nr), "num_entries %zu exceeds 2^%zu",
             num_entries, nr);
  PK_REQUIRE(out && aligned16(out), "out must be a 16-byte aligned device pointer");
  if (nr == 0) {  // eq over no variables is the single entry 1
    HostFr one = HostFr::one();
    PK_CUDA(cudaMemcpyAsync(out, one.l, 32, cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaStreamSynchronize(s));
    return PKG_OK;
  }
  int nhi = (int)(nr + 1) / 2, nlo = (int)nr - nhi;
  Scratch scr;
  size_t nh = size_t(1) << nhi, nl = size_t(1) << nlo;
  int rc = scr.alloc(32 * (nr + nh + nl), s);
  if (rc) return rc;
  uint64_t* d_r = static_cast<uint64_t*>(scr.ptr);
  uint64_t* d_hi = d_r + 4 * nr;
  uint64_t* d_lo = d_hi + 4 * nh;
  PK_CUDA(cudaMemcpyAsync(d_r, r_host, 32 * nr, cudaMemcpyHostToDevice, s));
  eq_small_kernel<<<ew_grid(nh), 256, 0, s>>>(d_r, nhi, d_hi);
  PK_CHECK_LAUNCH("eq_small_kernel");
  eq_small_kernel<<<ew_grid(nl), 256, 0, s>>>(d_r + 4 * nhi, nlo, d_lo);
  PK_CHECK_LAUNCH("eq_small_kernel");
  eq_combine_kernel<<<ew_grid(num_entries), 256, 0, s>>>(d_hi, d_lo, nlo, num_entries, out);
  PK_CHECK_LAUNCH("eq_combine_kernel");
  // a pinned r must outlive the async copy: callers whose r stays valid
  // until their next synchronisation pass sync = false
  if (sync) PK_CUDA(cudaStreamSynchronize(s));
  return PKG_OK;
}

// err: device word, zeroed by the caller before the launch.
int witness_bounds_device(const pkg_r1cs* r1cs, const uint64_t* w, size_t padded, uint64_t* ta,
                          uint64_t* tb, uint64_t* tc, uint32_t* err, cudaStream_t s) {
  if (padded == 0) return PKG_OK;
  PK_REQUIRE(aligned16(ta) && aligned16(tb) && aligned16(tc) && aligned16(w) &&
                 aligned16(r1cs->vals[0]) && aligned16(r1cs->vals[1]),
             "null or unaligned device pointer");
  witness_bounds_kernel<<<ew_grid(padded), 256, 0, s>>>(
      r1cs->row_ptr[0], r1cs->cols[0], r1cs->vals[0], r1cs->row_ptr[1], r1cs->cols[1],
      r1cs->vals[1], r1cs->num_constraints, r1cs->num_witnesses, padded, w, ta, tb, tc, err);
  PK_CHECK_LAUNCH("witness_bounds_kernel");
  return PKG_OK;
}

// Nonzeros from which the two balanced passes replace the one-row-per-thread
// kernel (below it the product temporary is not worth its traffic).
constexpr size_t kSpmvBalancedNnz = size_t(1) << 16;

// err: device word, zeroed by the caller before the launch.  nnz: the
// matrix's nonzero count (row_ptr[num_rows]), or 0 if the caller does not
// know it (one thread per row then).
int spmv_device(const uint64_t* row_ptr, const uint32_t* cols, const uint64_t* vals,
                size_t num_rows, size_t num_cols, const uint64_t* x, uint64_t* y, uint32_t* err,
                cudaStream_t s, size_t nnz) {
  if (num_rows == 0) return PKG_OK;
  PK_REQUIRE(row_ptr && y && aligned16(y) && aligned16(vals) && aligned16(x),
             "null or unaligned device pointer");
  // rows of at most ~one entry (a transposed C: one constraint per output
  // column) leave nothing to balance
  if (nnz < kSpmvBalancedNnz || nnz <= num_rows) {
    spmv_csr_kernel<<<ew_grid(num_rows), 256, 0, s>>>(row_ptr, cols, vals, num_rows, num_cols, x,
                                                     y, err);
    PK_CHECK_LAUNCH("spmv_csr_kernel");
    return PKG_OK;
  }
  Scratch tmp;
  int rc = tmp.alloc(32 * nnz, s);
  if (rc) return rc;
  uint64_t* prod = static_cast<uint64_t*>(tmp.ptr);
  spmv_products_kernel<<<ew_grid(nnz), 256, 0, s>>>(cols, vals, nnz, num_cols, x, prod, err);
  PK_CHECK_LAUNCH("spmv_products_kernel");
  spmv_rowsum_kernel<<<ew_grid(num_rows), 256, 0, s>>>(row_ptr, prod, num_rows, y);
  PK_CHECK_LAUNCH("spmv_rowsum_kernel");
  return PKG_OK;
}

static int read_err_flag(uint32_t* d_err, cudaStream_t s, const char* what) {
  uint32_t h = 0;
  PK_CUDA(cudaMemcpyAsync(&h, d_err, 4, cudaMemcpyDeviceToHost, s));
  PK_CUDA(cudaStreamSynchronize(s));
  if (h) {
    set_last_error("%s: column index out of range", what);
    return PKG_ERR_INVALID_ARGUMENT;
  }
  return PKG_OK;
}

int dot_device(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out, uint64_t* part,
               cudaStream_t s, unsigned* ticket) {
  PK_REQUIRE(ticket && out, "dot_device needs the thread's fused slots");
  dot_kernel<<<red_grid(n), kRedThreads, 0, s>>>(a, b, n,
                                                 RedOut{part, ticket, out, fused_next_seq()});
  PK_CHECK_LAUNCH("dot_kernel");
  return PKG_OK;
}

// ---- host transcript stand-in ------------------------------------------
struct HostTranscript {
  HostFr l, r;
  void init(const uint64_t domain[4]) {
    l = HostSky::reduce(HostFr::from_limbs(domain));
    r = HostFr::zero();
    HostSky::permute(l, r);
  }
  void absorb(const HostFr& x_mont) {
    l = HostFr::add(l, HostFr::from_mont(x_mont));
    HostSky::permute(l, r);
  }
  HostFr squeeze() {
    HostSky::permute(l, r);
    return HostFr::to_mont(l);
  }
};

static HostFr eval_cubic(const HostFr* c, const HostFr& x) {
  HostFr acc = HostFr::mul(x, c[3]);
  acc = HostFr::mul(HostFr::add(acc, c[2]), x);
  acc = HostFr::mul(HostFr::add(acc, c[1]), x);
  return HostFr::add(acc, c[0]);
}

// 1/2 in Montgomery form, inverted once (an inversion is ~400 products).
static const HostFr& half_mont() {
  static const HostFr h = HostFr::inv(HostFr::add(HostFr::one(), HostFr::one()));
  return h;
}

// g_i(0) + g_i(1) of one blinding cubic
static HostFr cubic_sum01(const HostFr* c) {
  return HostFr::add(eval_cubic(c, HostFr::zero()), eval_cubic(c, HostFr::one()));
}

// The coefficients of compute_blinding_coefficients_for_round for
// cf < n from its two sums: prefix = sum_{i < cf} g_i(alpha_i), suffix =
// sum_{i > cf} (g_i(0) + g_i(1)).
static void blinding_from_sums(const HostFr* g, size_t n, size_t cf, const HostFr& prefix,
                               const HostFr& suffix, HostFr res[4]) {
  HostFr pm = HostFr::one();
  for (size_t i = 0; i < n - 1 - cf; i++) pm = HostFr::add(pm, pm);
  HostFr sm = HostFr::mul(pm, half_mont());
  HostFr cst = HostFr::add(HostFr::mul(pm, prefix), HostFr::mul(sm, suffix));
  const HostFr* cur = g + 4 * cf;
  res[0] = HostFr::add(HostFr::mul(pm, cur[0]), cst);
  for (int k = 1; k < 4; k++) res[k] = HostFr::mul(pm, cur[k]);
}

// compute_blinding_coefficients_for_round (whir_r1cs.rs:427-492)
static void blinding_coeffs(const HostFr* g, size_t n, size_t compute_for, const HostFr* alphas,
                            HostFr out[4]) {
  bool all_fixed = false;
  size_t cf = compute_for;
  if (cf == n) {
    all_fixed = true;
    cf = n - 1;
  }
  HostFr prefix = HostFr::zero(), suffix = HostFr::zero();
  for (size_t i = 0; i < cf; i++) prefix = HostFr::add(prefix, eval_cubic(g + 4 * i, alphas[i]));
  for (size_t i = cf + 1; i < n; i++) suffix = HostFr::add(suffix, cubic_sum01(g + 4 * i));
  if (!all_fixed) {
    blinding_from_sums(g, n, cf, prefix, suffix, out);
    return;
  }
  HostFr pm = HostFr::one();
  for (size_t i = 0; i < n - 1 - cf; i++) pm = HostFr::add(pm, pm);
  HostFr sm = HostFr::mul(pm, half_mont());
  HostFr cst = HostFr::add(HostFr::mul(pm, prefix), HostFr::mul(sm, suffix));
  const HostFr* cur = g + 4 * cf;
  HostFr res[4] = {HostFr::add(HostFr::mul(pm, cur[0]), cst), HostFr::mul(pm, cur[1]),
                   HostFr::mul(pm, cur[2]), HostFr::mul(pm, cur[3])};
  if (all_fixed) {
    out[0] = eval_cubic(res, alphas[cf]);
    out[1] = out[2] = out[3] = HostFr::zero();
    return;
  }
  for (int k = 0; k < 4; k++) out[k] = res[k];
}

// Tables of at most this many entries finish their rounds on the host.
constexpr size_t kHostTailEntries = 64;

// spartan_round_kernel on host tables: with fold, bind the top variable
// first (t[j] += fold (t[j + size/2] - t[j])) and halve size; then the sums
// f(0), f(-1), f(inf) over the pairs (j, j + size/2) (whir_r1cs.rs:552-558),
// as canonical Montgomery limbs into out.
static void host_spartan_round(std::vector<HostFr> (&t)[4], size_t size, const HostFr* fold,
                               uint64_t out[12]) {
  if (fold) {
    const size_t h = size / 2;
    for (auto& v : t)
      for (size_t j = 0; j < h; j++) v[j] = HostFr::add(v[j], HostFr::mul(*fold, HostFr::sub(v[j + h], v[j])));
    size = h;
  }
  const size_t q = size / 2;
  HostFr f0 = HostFr::zero(), fm1 = HostFr::zero(), finf = HostFr::zero();
  for (size_t j = 0; j < q; j++) {
    const HostFr a0 = t[0][j], a1 = t[0][j + q], b0 = t[1][j], b1 = t[1][j + q];
    const HostFr c0 = t[2][j], c1 = t[2][j + q], e0 = t[3][j], e1 = t[3][j + q];
    f0 = HostFr::add(f0, HostFr::mul(e0, HostFr::sub(HostFr::mul(a0, b0), c0)));
    const HostFr a2 = HostFr::sub(HostFr::add(a0, a0), a1), b2 = HostFr::sub(HostFr::add(b0, b0), b1);
    const HostFr c2 = HostFr::sub(HostFr::add(c0, c0), c1), e2 = HostFr::sub(HostFr::add(e0, e0), e1);
    fm1 = HostFr::add(fm1, HostFr::mul(e2, HostFr::sub(HostFr::mul(a2, b2), c2)));
    finf = HostFr::add(finf, HostFr::mul(HostFr::sub(e1, e0),
                                         HostFr::mul(HostFr::sub(a1, a0), HostFr::sub(b1, b0))));
  }
  memcpy(out, f0.l, 32);
  memcpy(out + 4, fm1.l, 32);
  memcpy(out + 8, finf.l, 32);
}

}  // namespace pk

using namespace pk;

static_assert(sizeof(pkg_transcript) == 64, "transcript state is two field elements");

extern "C" int pkg_transcript_init(pkg_transcript* t, const uint64_t domain[4]) {
  PK_REQUIRE(t && domain, "null pointer");
  HostTranscript ht;
  ht.init(domain);
  memcpy(t->l, ht.l.l, 32);
  memcpy(t->r, ht.r.l, 32);
  return PKG_OK;
}

extern "C" int pkg_transcript_absorb(pkg_transcript* t, const uint64_t x[4]) {
  PK_REQUIRE(t && x, "null pointer");
  HostTranscript ht;
  ht.l = HostFr::from_limbs(t->l);
  ht.r = HostFr::from_limbs(t->r);
  ht.absorb(HostFr::from_limbs(x));
  memcpy(t->l, ht.l.l, 32);
  memcpy(t->r, ht.r.l, 32);
  return PKG_OK;
}

extern "C" int pkg_transcript_squeeze_bytes(pkg_transcript* t, uint8_t* out, size_t n) {
  PK_REQUIRE(t && (out || n == 0), "null pointer");
  HostTranscript ht;
  ht.l = HostFr::from_limbs(t->l);
  ht.r = HostFr::from_limbs(t->r);
  for (size_t done = 0; done < n;) {
    const HostFr c = HostFr::from_mont(ht.squeeze());
    const size_t take = std::min<size_t>(31, n - done);
    for (size_t i = 0; i < take; i++) out[done + i] = (uint8_t)(c.l[i / 8] >> (8 * (i % 8)));
    done += take;
  }
  memcpy(t->l, ht.l.l, 32);
  memcpy(t->r, ht.r.l, 32);
  return PKG_OK;
}

extern "C" int pkg_transcript_squeeze(pkg_transcript* t, uint64_t out[4]) {
  PK_REQUIRE(t && out, "null pointer");
  HostTranscript ht;
  ht.l = HostFr::from_limbs(t->l);
  ht.r = HostFr::from_limbs(t->r);
  HostFr v = ht.squeeze();
  memcpy(out, v.l, 32);
  memcpy(t->l, ht.l.l, 32);
  memcpy(t->r, ht.r.l, 32);
  return PKG_OK;
}

extern "C" int pkg_spartan_round(uint64_t* a, uint64_t* b, uint64_t* c, uint64_t* eq, size_t size,
                                 const uint64_t* fold, uint64_t out[12], pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(size) && size >= 2, "table size %zu must be a power of two >= 2", size);
  PK_REQUIRE(!fold || size >= 4, "folding needs size >= 4 (got %zu)", size);
  PK_REQUIRE(a && b && c && eq && out, "null pointer");
  PK_REQUIRE(aligned16(a) && aligned16(b) && aligned16(c) && aligned16(eq),
             "device buffers must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  rc = spartan_round_device(a, b, c, eq, size, fold, fs.part, fs.dev, s, fs.ticket);
  if (rc) return rc;
  return fused_read(out, fs, 96, s);
}

extern "C" int pkg_eq_hypercube(const uint64_t* r, size_t nr, size_t num_entries, uint64_t* out,
                                pkg_stream_t stream) {
  return eq_hypercube_device(r, nr, num_entries, out, as_stream(stream), true);
}

extern "C" int pkg_spmv_csr(const uint64_t* row_ptr, const uint32_t* cols, const uint64_t* vals,
                            size_t num_rows, size_t num_cols, const uint64_t* x, uint64_t* y,
                            pkg_stream_t stream) {
  if (num_rows == 0) return PKG_OK;
  cudaStream_t s = as_stream(stream);
  Scratch scr;
  int rc = scr.alloc(256, s);
  if (rc) return rc;
  uint32_t* err = static_cast<uint32_t*>(scr.ptr);
  PK_CUDA(cudaMemsetAsync(err, 0, 4, s));
  PK_REQUIRE(row_ptr, "null row pointers");
  uint64_t nnz = 0;  // row_ptr[num_rows], for the balanced passes
  if ((rc = read_small(&nnz, row_ptr + num_rows, 8, s))) return rc;
  PK_REQUIRE(nnz < (uint64_t(1) << 40), "row_ptr[num_rows] = %llu is not a nonzero count",
             (unsigned long long)nnz);
  rc = spmv_device(row_ptr, cols, vals, num_rows, num_cols, x, y, err, s, (size_t)nnz);
  if (rc) return rc;
  return read_err_flag(err, s, "pkg_spmv_csr");
}

extern "C" int pkg_hadamard_pad(const uint64_t* a, const uint64_t* b, size_t n, size_t padded,
                                uint64_t* c, pkg_stream_t stream) {
  PK_REQUIRE(padded >= n, "padded length %zu < n %zu", padded, n);
  if (padded == 0) return PKG_OK;
  PK_REQUIRE(c && aligned16(c) && aligned16(a) && aligned16(b), "null or unaligned pointer");
  cudaStream_t s = as_stream(stream);
  hadamard_pad_kernel<<<ew_grid(padded), 256, 0, s>>>(a, b, n, padded, c);
  PK_CHECK_LAUNCH("hadamard_pad_kernel");
  return PKG_OK;
}

extern "C" int pkg_dot(const uint64_t* a, const uint64_t* b, size_t n, uint64_t out[4],
                       pkg_stream_t stream) {
  PK_REQUIRE(out, "null output");
  if (n == 0) {
    memset(out, 0, 32);
    return PKG_OK;
  }
  PK_REQUIRE(a && b && aligned16(a) && aligned16(b), "null or unaligned pointer");
  cudaStream_t s = as_stream(stream);
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  rc = dot_device(a, b, n, fs.dev, fs.part, s, fs.ticket);
  if (rc) return rc;
  return fused_read(out, fs, 32, s);
}

extern "C" int pkg_csr_transpose(const uint64_t* row_ptr, const uint32_t* cols, const uint64_t* vals,
                                 size_t num_rows, size_t num_cols, size_t nnz,
                                 uint64_t* row_ptr_t, uint32_t* cols_t, uint64_t* vals_t,
                                 pkg_stream_t stream) {
  PK_REQUIRE(row_ptr && row_ptr_t, "null row pointer array");
  PK_REQUIRE(num_cols < (size_t(1) << 32) && num_rows < (size_t(1) << 32),
             "matrix dimensions must fit u32 column indices");
  cudaStream_t s = as_stream(stream);
  Scratch scr;
  // counts (u32, num_cols), cursor (u64, num_cols + 1), cub temp
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (unsigned long long*)nullptr,
                                (unsigned long long*)nullptr, (int)(num_cols + 1), s);
  size_t counts_bytes = ((4 * num_cols + 255) / 256) * 256;
  size_t wide_bytes = ((8 * (num_cols + 1) + 255) / 256) * 256;
  int rc = scr.alloc(counts_bytes + wide_bytes + cub_bytes + 512, s);
  if (rc) return rc;
  uint8_t* base = static_cast<uint8_t*>(scr.ptr);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base);
  unsigned long long* wide = reinterpret_cast<unsigned long long*>(base + counts_bytes);
  void* cub_tmp = base + counts_bytes + wide_bytes;
  uint32_t* err = reinterpret_cast<uint32_t*>(base + counts_bytes + wide_bytes + ((cub_bytes + 255) / 256) * 256);
  PK_CUDA(cudaMemsetAsync(err, 0, 4, s));
  PK_CUDA(cudaMemsetAsync(counts, 0, 4 * num_cols, s));
  PK_CUDA(cudaMemsetAsync(wide, 0, 8 * (num_cols + 1), s));
  if (nnz) {
    csr_count_cols_kernel<<<ew_grid(nnz), 256, 0, s>>>(cols, nnz, num_cols, counts, err);
    PK_CHECK_LAUNCH("csr_count_cols_kernel");
  }
  if (num_cols) {
    widen_kernel<<<ew_grid(num_cols), 256, 0, s>>>(counts, num_cols, wide);
    PK_CHECK_LAUNCH("widen_kernel");
  }
  PK_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, wide,
                                        reinterpret_cast<unsigned long long*>(row_ptr_t),
                                        (int)(num_cols + 1), s));
  count_launch();
  // cursor = row_ptr_t[0..num_cols) (reuse `wide`)
  PK_CUDA(cudaMemcpyAsync(wide, row_ptr_t, 8 * (num_cols + 1), cudaMemcpyDeviceToDevice, s));
  if (nnz && num_rows) {
    csr_scatter_kernel<<<ew_grid(num_rows), 256, 0, s>>>(row_ptr, cols, vals, num_rows, num_cols,
                                                         wide, cols_t, vals_t);
    PK_CHECK_LAUNCH("csr_scatter_kernel");
  }
  return read_err_flag(err, s, "pkg_csr_transpose");
}

extern "C" int pkg_spartan_sumcheck(uint64_t* a, uint64_t* b, uint64_t* c, size_t m0,
                                    const uint64_t* g, const uint64_t* w1_blinding,
                                    pkg_transcript* transcript, uint64_t* r_out, uint64_t rho_out[4],
                                    uint64_t sum_g_out[4], uint64_t* coeffs_out,
                                    uint64_t* alpha_out, uint64_t blinding_eval[4],
                                    pkg_stream_t stream) {
  PK_REQUIRE(m0 >= 1 && m0 <= 30, "m0 %zu out of range [1, 30]", m0);
  PK_REQUIRE(a && b && c && g && w1_blinding && transcript && r_out && rho_out && sum_g_out &&
                 coeffs_out && alpha_out && blinding_eval,
             "null pointer");
  PK_REQUIRE(aligned16(a) && aligned16(b) && aligned16(c), "device buffers must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  const size_t n = size_t(1) << m0;
  HostTranscript t;
  t.l = HostFr::from_limbs(transcript->l);
  t.r = HostFr::from_limbs(transcript->r);
  std::vector<HostFr> r(m0), alpha(m0), gv(4 * m0);
  for (size_t i = 0; i < 4 * m0; i++) gv[i] = HostFr::from_limbs(g + 4 * i);
  for (size_t i = 0; i < m0; i++) {  // whir_r1cs.rs:529
    r[i] = t.squeeze();
    memcpy(r_out + 4 * i, r[i].l, 32);
  }
  // scratch: eq table (n Fr), partials; each round's sums go to the
  // thread's fused slots
  const int gmax = red_grid(n / 2);
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  Scratch scr;
  if ((rc = scr.alloc(32 * (n + 3 * (size_t)gmax), s))) return rc;
  uint64_t* eq = static_cast<uint64_t*>(scr.ptr);
  uint64_t* part = eq + 4 * n;
  rc = eq_hypercube_device(r_out, m0, n, eq, s, false);  // :530; the rounds synchronise
  if (rc) return rc;
  HostFr g0[4];
  blinding_coeffs(gv.data(), m0, 0, nullptr, g0);  // sum_over_hypercube, :494-501
  HostFr sum_g = HostFr::add(eval_cubic(g0, HostFr::zero()), eval_cubic(g0, HostFr::one()));
  memcpy(sum_g_out, sum_g.l, 32);
  t.absorb(sum_g);                  // :541
  HostFr rho = t.squeeze();         // :543
  memcpy(rho_out, rho.l, 32);
  HostFr saved = HostFr::mul(rho, sum_g);
  const HostFr half = half_mont();
  size_t size = n;
  uint64_t h[12];
  // the blinding coefficients' two sums, kept as running sums over the rounds
  HostFr bprefix = HostFr::zero(), bsuffix = HostFr::zero();
  for (size_t i = 1; i < m0; i++) bsuffix = HostFr::add(bsuffix, cubic_sum01(&gv[4 * i]));
  // the last rounds, on tables of at most kHostTailEntries, run on the host
  // (a device round there is launch and round-trip latency)
  std::vector<HostFr> tab[4];
  bool on_host = false;
  for (size_t idx = 0; idx < m0; idx++) {  // :550-610
    if (!on_host && size <= kHostTailEntries) {
      for (int k = 0; k < 4; k++) tab[k].resize(size);
      const HostRead reads[4] = {{tab[0][0].l, a, 32 * size}, {tab[1][0].l, b, 32 * size},
                                 {tab[2][0].l, c, 32 * size}, {tab[3][0].l, eq, 32 * size}};
      if ((rc = read_small(reads, 4, s))) return rc;
      on_host = true;
    }
    if (on_host) {
      host_spartan_round(tab, size, idx ? &alpha[idx - 1] : nullptr, h);
    } else {
      rc = spartan_round_device(a, b, c, eq, size, idx ? alpha[idx - 1].l : nullptr, part, fs.dev,
                                s, fs.ticket);
      if (rc) return rc;
      if ((rc = fused_read(h, fs, 96, s))) return rc;
    }
    if (idx) size /= 2;
    HostFr gp[4];
    if (idx) {
      bprefix = HostFr::add(bprefix, eval_cubic(&gv[4 * (idx - 1)], alpha[idx - 1]));
      bsuffix = HostFr::sub(bsuffix, cubic_sum01(&gv[4 * idx]));
    }
    blinding_from_sums(gv.data(), m0, idx, bprefix, bsuffix, gp);
    HostFr h0 = HostFr::from_limbs(h), hem1 = HostFr::from_limbs(h + 4),
           hinf = HostFr::from_limbs(h + 8);
    HostFr cf[4];
    cf[0] = HostFr::add(h0, HostFr::mul(rho, gp[0]));
    HostFr gem1 = HostFr::sub(HostFr::add(HostFr::sub(gp[0], gp[1]), gp[2]), gp[3]);
    HostFr cem1 = HostFr::add(hem1, HostFr::mul(rho, gem1));
    cf[2] = HostFr::mul(half, HostFr::sub(HostFr::sub(HostFr::sub(HostFr::add(saved, cem1), cf[0]),
                                                      cf[0]),
                                          cf[0]));
    cf[3] = HostFr::add(hinf, HostFr::mul(rho, gp[3]));
    cf[1] = HostFr::sub(HostFr::sub(HostFr::sub(HostFr::sub(saved, cf[0]), cf[0]), cf[3]), cf[2]);
    for (int k = 0; k < 4; k++) {
      memcpy(coeffs_out + 16 * idx + 4 * k, cf[k].l, 32);
      t.absorb(cf[k]);
    }
    alpha[idx] = t.squeeze();
    memcpy(alpha_out + 4 * idx, alpha[idx].l, 32);
    saved = eval_cubic(cf, alpha[idx]);
  }
  // blinding_eval = <expand_powers::<4>(alpha), w1[offset..offset + 4*m0]> (:613-618)
  HostFr acc = HostFr::zero();
  for (size_t i = 0; i < m0; i++) {
    HostFr pw = HostFr::one();
    for (int k = 0; k < 4; k++) {
      acc = HostFr::add(acc, HostFr::mul(pw, HostFr::from_limbs(w1_blinding + 4 * (4 * i + k))));
      pw = HostFr::mul(pw, alpha[i]);
    }
  }
  memcpy(blinding_eval, acc.l, 32);
  t.absorb(acc);  // prover_message(&blinding_eval), :618
  memcpy(transcript->l, t.l.l, 32);
  memcpy(transcript->r, t.r.l, 32);
  return PKG_OK;
}

namespace {
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

extern "C" size_t pkg_r1cs_transposes_bytes(const pkg_r1cs* r1cs) {
  if (!r1cs) return 0;
  size_t total = 0;
  for (int k = 0; k < 3; k++) {
    const size_t nnz = r1cs->nnz[k] ? r1cs->nnz[k] : 1;
    total += align256(8 * (r1cs->num_witnesses + 1)) + align256(4 * nnz) + align256(32 * nnz);
  }
  return total;
}

extern "C" int pkg_r1cs_build_transposes(pkg_r1cs* r1cs, void* buf, pkg_stream_t stream) {
  PK_REQUIRE(r1cs && buf, "null pointer");
  PK_REQUIRE((reinterpret_cast<uintptr_t>(buf) & 255) == 0, "buffer must be 256-byte aligned");
  uint8_t* at = static_cast<uint8_t*>(buf);
  const size_t nw = r1cs->num_witnesses, nc = r1cs->num_constraints;
  for (int k = 0; k < 3; k++) {
    const size_t nnz = r1cs->nnz[k] ? r1cs->nnz[k] : 1;
    uint64_t* rp = reinterpret_cast<uint64_t*>(at);
    at += align256(8 * (nw + 1));
    uint32_t* cl = reinterpret_cast<uint32_t*>(at);
    at += align256(4 * nnz);
    uint64_t* vl = reinterpret_cast<uint64_t*>(at);
    at += align256(32 * nnz);
    const int rc = pkg_csr_transpose(r1cs->row_ptr[k], r1cs->cols[k], r1cs->vals[k], nc, nw,
                                     r1cs->nnz[k], rp, cl, vl, stream);
    if (rc) return rc;
    r1cs->row_ptr_t[k] = rp;
    r1cs->cols_t[k] = cl;
    r1cs->vals_t[k] = vl;
  }
  return PKG_OK;
}
