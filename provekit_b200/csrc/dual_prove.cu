// dual_prove.cu -- the dual-commitment proof of an R1CS with verifier
// challenges: Prove::prove's two commitments (provekit/prover/src/lib.rs:145-232)
// and prove_from_alphas's second branch (provekit/prover/src/whir_r1cs.rs:302-425),
// split at the point where the caller solves w2 from the challenges.
//
// Device data held between the two calls (one pool allocation): the whole
// witness (w1 copied at begin, w2 at finish), and per commitment its padded
// polynomial batch (2^m Fr, plus the whir-ZK mask), RS codeword and Merkle
// layers.  finish adds the sumcheck tables, eq(alpha), the transposed
// products and the two statement sets as scratch.  The host keeps the
// transcript, as on the single-commitment path.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "fr_host.hpp"
#include "internal.cuh"
#include "pk_common.cuh"
#include "rs_internal.cuh"

struct pkg_dual_prove {
  pkg_r1cs r1cs{};
  size_t w1_size = 0, nw = 0, nc = 0, np = 0, m = 0, m0 = 0;
  std::vector<size_t> offsets;
  pkg_whir_params whir{};
  uint64_t blinding_seed = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  bool finished = false;
  void* mem = nullptr;  // the allocation below, from the library pool
  uint64_t *witness = nullptr, *poly[2] = {nullptr, nullptr}, *cw[2] = {nullptr, nullptr};
  uint8_t* layers[2] = {nullptr, nullptr};
  std::vector<uint64_t> g;  // the blinding univariates (4 m0 Fr)
  uint64_t ood[2][4 * 5] = {};
  pkg_transcript t{};
  uint8_t root1[32] = {};
};

namespace pk {
namespace {

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// The commitment's sizes: polynomial batch, codeword and layers (bytes).
struct CommitSizes {
  size_t n, cw_len, poly_bytes, cw_bytes, layer_bytes;
  explicit CommitSizes(const pkg_whir_params& w) {
    n = size_t(1) << w.num_variables;
    cw_len = (n >> w.folding_factor) << w.log_inv_rate;
    poly_bytes = round256(32 * n * w.batch_size);
    cw_bytes = round256(32 * (size_t(1) << w.folding_factor) * w.batch_size * cw_len);
    layer_bytes = round256(32 * (2 * cw_len - 1));
  }
};

// One part's commitment (whir_r1cs.rs commit, :82-140): vals (device, nvals
// Fr) padded to 2^m, g at g_offset when given, the mask polynomial for
// whir-ZK; RS encode, tree, then the root and OOD samples into the
// transcript (pkg_whir_commit_ood).
int commit_part(pkg_dual_prove* st, int k, const uint64_t* vals, size_t nvals, const uint64_t* g,
                size_t g_offset, uint64_t mask_seed, uint64_t* commit_words) {
  const pkg_whir_params& w = st->whir;
  const CommitSizes cs(w);
  const size_t M = size_t(1) << w.folding_factor, L = cs.n >> w.folding_factor;
  cudaStream_t s = st->stream;
  uint64_t* poly = st->poly[k];
  PK_CUDA(cudaMemsetAsync(poly, 0, 32 * cs.n, s));
  if (nvals) PK_CUDA(cudaMemcpyAsync(poly, vals, 32 * nvals, cudaMemcpyDeviceToDevice, s));
  if (g)
    PK_CUDA(cudaMemcpyAsync(poly + 4 * g_offset, g, 32 * 4 * st->m0, cudaMemcpyHostToDevice, s));
  int rc;
  if (w.batch_size == 2 &&
      (rc = pkg_sample_fr_indexed(st->blinding_seed ^ mask_seed, 0, cs.n, poly + 4 * cs.n,
                                  reinterpret_cast<pkg_stream_t>(s))))
    return rc;
  if ((rc = rs_encode_device(poly, M * w.batch_size, L, nullptr, 0, cs.cw_len, st->cw[k], s)))
    return rc;
  if ((rc = merkle_tree_fr_device(st->cw[k], M * w.batch_size, cs.cw_len, PKG_LEAF_CANONICAL,
                                  st->layers[k], s)))
    return rc;
  return pkg_whir_commit_ood(&w, &st->t, poly, st->layers[k], commit_words, st->ood[k],
                             reinterpret_cast<pkg_stream_t>(s));
}

// dst[idx[j]] = vals[j] over k distinct indices (the challenge weight).
__global__ void scatter_fr_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ idx,
                                  const uint64_t* __restrict__ vals, size_t k) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < k;
       j += (size_t)gridDim.x * blockDim.x) {
    const size_t at = idx[j];
    for (int q = 0; q < 4; q++) dst[4 * at + q] = vals[4 * j + q];
  }
}

void free_state(pkg_dual_prove* st) {
  if (!st) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(st->device);
  if (st->mem) {
    cudaFreeAsync(st->mem, st->stream);
    cudaStreamSynchronize(st->stream);
  }
  cudaGetLastError();
  if (prev >= 0) cudaSetDevice(prev);
  delete st;
}

}  // namespace
}  // namespace pk

using namespace pk;

extern "C" int pkg_r1cs_sizing_split(size_t num_constraints, size_t num_witnesses,
                                     size_t w1_size, size_t* m_out, size_t* m0_out) {
  PK_REQUIRE(m_out && m0_out, "null output");
  PK_REQUIRE(num_constraints >= 1 && num_witnesses >= 1, "empty R1CS");
  PK_REQUIRE(w1_size >= 1 && w1_size <= num_witnesses, "w1_size %zu outside 1..%zu", w1_size,
             num_witnesses);
  const size_t m1 = log2_exact(w1_size), m2 = log2_exact(num_witnesses - w1_size);
  size_t m = m1 > m2 ? m1 : m2, m0 = log2_exact(num_constraints);
  if (m < 13) m = 13;  // MIN_WHIR_NUM_VARIABLES
  if (m0 < 1) m0 = 1;  // MIN_SUMCHECK_NUM_VARIABLES
  if ((size_t(1) << m) - w1_size < 4 * m0) m++;
  *m_out = m;
  *m0_out = m0;
  return PKG_OK;
}

extern "C" void pkg_dual_prove_free(pkg_dual_prove* state) { free_state(state); }

extern "C" int pkg_dual_prove_begin(const pkg_r1cs* r1cs, size_t w1_size,
                                    const size_t* challenge_offsets, size_t num_challenges,
                                    const uint64_t* w1, uint64_t blinding_seed,
                                    uint64_t transcript_domain, const pkg_whir_params* whir,
                                    uint64_t* whir_commit_words1, uint64_t* challenges,
                                    pkg_dual_prove** state, pkg_stream_t stream) {
  PK_REQUIRE(state, "null state output");
  *state = nullptr;
  PK_REQUIRE(r1cs && w1 && whir && whir_commit_words1, "null pointer");
  PK_REQUIRE(num_challenges == 0 || (challenge_offsets && challenges),
             "null challenge offsets or output");
  PK_REQUIRE(aligned16(w1), "w1 must be 16-byte aligned");
  const size_t nc = r1cs->num_constraints, nw = r1cs->num_witnesses;
  size_t m = 0, m0 = 0;
  int rc = pkg_r1cs_sizing_split(nc, nw, w1_size, &m, &m0);
  if (rc) return rc;
  PK_REQUIRE(m0 <= 30 && m <= 28, "instance too large (m=%zu, m0=%zu)", m, m0);
  PK_REQUIRE(r1cs->num_public_inputs + 1 <= w1_size, "%zu public inputs but w1 holds %zu",
             r1cs->num_public_inputs, w1_size);
  PK_REQUIRE(pkg_whir_proof_words(whir, 3) != 0, "invalid WHIR parameters");
  PK_REQUIRE(whir->num_variables == m, "WHIR parameters for %u variables, the R1CS needs %zu",
             whir->num_variables, m);
  PK_REQUIRE(whir->batch_size == 1 || whir->batch_size == 2,
             "WHIR batch of %u: each part is committed alone or with one mask polynomial",
             whir->batch_size);
  for (size_t j = 0; j < num_challenges; j++)  // SparseCovector::new (prefix_covector.rs:257-266)
    PK_REQUIRE(challenge_offsets[j] < (size_t(1) << m), "challenge offset %zu outside 2^%zu",
               challenge_offsets[j], m);

  pkg_dual_prove* st = new (std::nothrow) pkg_dual_prove;
  PK_REQUIRE(st, "out of host memory");
  st->r1cs = *r1cs;
  st->w1_size = w1_size;
  st->nw = nw;
  st->nc = nc;
  st->np = r1cs->num_public_inputs;
  st->m = m;
  st->m0 = m0;
  st->offsets.assign(challenge_offsets, challenge_offsets + num_challenges);
  st->whir = *whir;
  st->blinding_seed = blinding_seed;
  st->stream = as_stream(stream);
  cudaGetDevice(&st->device);
  const CommitSizes cs(*whir);
  const size_t wit_bytes = round256(32 * nw);
  const size_t part = cs.poly_bytes + cs.cw_bytes + cs.layer_bytes;
  cudaMemPool_t pool = lib_pool();
  if (!pool) {
    free_state(st);
    set_last_error("could not create the library memory pool");
    return PKG_ERR_CUDA;
  }
  cudaError_t e = cudaMallocFromPoolAsync(&st->mem, wit_bytes + 2 * part, pool, st->stream);
  if (e != cudaSuccess) {
    st->mem = nullptr;
    free_state(st);
    return cuda_status(e, "cudaMallocFromPoolAsync");
  }
  uint8_t* base = static_cast<uint8_t*>(st->mem);
  st->witness = reinterpret_cast<uint64_t*>(base);
  for (int k = 0; k < 2; k++) {
    uint8_t* p = base + wit_bytes + k * part;
    st->poly[k] = reinterpret_cast<uint64_t*>(p);
    st->cw[k] = reinterpret_cast<uint64_t*>(p + cs.poly_bytes);
    st->layers[k] = p + cs.poly_bytes + cs.cw_bytes;
  }
  auto fail = [st](int code) {
    free_state(st);
    return code;
  };
  if (cudaMemcpyAsync(st->witness, w1, 32 * w1_size, cudaMemcpyDeviceToDevice, st->stream) !=
      cudaSuccess)
    return fail(cuda_status(cudaGetLastError(), "cudaMemcpyAsync(w1)"));
  const uint64_t dom[4] = {transcript_domain, 0, 0, 0};
  pkg_transcript_init(&st->t, dom);
  // w1's commitment with the blinding univariates g at w1_size (lib.rs:184-187)
  st->g.resize(16 * m0);
  pkg_sample_fr(blinding_seed, 4 * m0, st->g.data(), 1);  // generate_blinding_univariates, seeded
  if ((rc = commit_part(st, 0, w1, w1_size, st->g.data(), w1_size, kMaskSeed, whir_commit_words1)))
    return fail(rc);
  memcpy(st->root1, whir_commit_words1, 32);
  // the challenges, squeezed in order (WitnessBuilder::Challenge, witness_builder.rs:167-170)
  for (size_t j = 0; j < num_challenges; j++) pkg_transcript_squeeze(&st->t, challenges + 4 * j);
  *state = st;
  return PKG_OK;
}

extern "C" int pkg_dual_prove_finish(pkg_dual_prove* st, const uint64_t* w2, pkg_dual_proof* out,
                                     uint64_t* whir_commit_words2, uint64_t* whir_proof1,
                                     uint64_t* whir_proof2) {
  PK_REQUIRE(st, "null state");
  PK_REQUIRE(!st->finished, "the state's proof was already finished");
  PK_REQUIRE(out && whir_commit_words2 && whir_proof1 && whir_proof2, "null output");
  const size_t w1_size = st->w1_size, nw = st->nw, nc = st->nc, np = st->np, m0 = st->m0;
  const size_t w2_size = nw - w1_size, nchal = st->offsets.size();
  PK_REQUIRE(w2 || w2_size == 0, "null w2");
  PK_REQUIRE(!w2 || aligned16(w2), "w2 must be 16-byte aligned");
  int cur = -1;
  PK_CUDA(cudaGetDevice(&cur));
  PK_REQUIRE(cur == st->device, "the state belongs to device %d, device %d is current",
             st->device, cur);
  st->finished = true;
  memset(out, 0, sizeof *out);
  pkg_spartan_proof* sp = &out->spartan;
  sp->m = st->m;
  sp->m0 = m0;
  memcpy(sp->root, st->root1, 32);
  cudaStream_t s = st->stream;
  const pkg_r1cs* r1cs = &st->r1cs;
  const CommitSizes cs(st->whir);
  const size_t n = cs.n, n0 = size_t(1) << m0;
  int rc;

  // w2 into the whole witness and its commitment (no blinding polynomial)
  if (w2_size)
    PK_CUDA(cudaMemcpyAsync(st->witness + 4 * w1_size, w2, 32 * w2_size, cudaMemcpyDeviceToDevice,
                            s));
  if ((rc = commit_part(st, 1, w2, w2_size, nullptr, 0, kMaskSeed2, whir_commit_words2)))
    return rc;
  memcpy(out->root2, whir_commit_words2, 32);

  // witness bounds over the whole witness and the zk sumcheck with w1's
  // blinding (prove_noir, whir_r1cs.rs:143-187)
  const size_t nparts = 4 * (size_t)sm_count();
  Scratch s_tab, s_misc, s_eq, s_alph, s_st;
  if ((rc = s_tab.alloc(32 * 3 * n0, s))) return rc;
  if ((rc = s_misc.alloc(256 + 32 * nparts, s))) return rc;
  uint64_t* ta = static_cast<uint64_t*>(s_tab.ptr);
  uint64_t* tb = ta + 4 * n0;
  uint64_t* tc = tb + 4 * n0;
  uint32_t* err = static_cast<uint32_t*>(s_misc.ptr);
  uint64_t* part = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(s_misc.ptr) + 256);
  PK_CUDA(cudaMemsetAsync(err, 0, 4, s));
  if ((rc = witness_bounds_device(r1cs, st->witness, n0, ta, tb, tc, err, s))) return rc;
  rc = pkg_spartan_sumcheck(ta, tb, tc, m0, st->g.data(), st->g.data(), &st->t, &sp->r[0][0],
                            sp->rho, sp->sum_g, &sp->coeffs[0][0], &sp->alpha[0][0],
                            sp->blinding_eval, reinterpret_cast<pkg_stream_t>(s));
  if (rc) return rc;
  uint32_t h_err = 0;
  if ((rc = read_small(&h_err, err, 4, s))) return rc;
  PK_REQUIRE(!h_err, "R1CS column index out of range");

  // eq(alpha), the public weights, the transposed products split at w1_size
  // (whir_r1cs.rs:311-326) and the statements of both WHIR proofs
  const size_t base = np ? 1 : 0, ncov1 = base + 4, ncov2 = 3 + (nchal ? 1 : 0);
  if ((rc = s_eq.alloc(32 * nc, s))) return rc;
  if ((rc = s_alph.alloc(32 * nw, s))) return rc;
  if ((rc = s_st.alloc(32 * (ncov1 + ncov2) * n, s))) return rc;
  uint64_t* eq = static_cast<uint64_t*>(s_eq.ptr);
  uint64_t* alph = static_cast<uint64_t*>(s_alph.ptr);
  uint64_t* st1 = static_cast<uint64_t*>(s_st.ptr);
  uint64_t* st2 = st1 + 4 * ncov1 * n;
  PK_CUDA(cudaMemsetAsync(st1, 0, 32 * (ncov1 + ncov2) * n, s));
  if ((rc = eq_hypercube_device(&sp->alpha[0][0], m0, nc, eq, s, false))) return rc;
  std::vector<uint64_t> pubw(4 * (np + 1));
  if ((rc = public_challenge(st->witness, np, pubw.data(), &st->t, sp->public_hash, sp->public_x,
                             s)))
    return rc;
  // the challenge weight x^j at offsets[j] (make_challenge_weight,
  // prefix_covector.rs:311-323), repeated offsets summed on the host
  std::vector<uint64_t> cidx, cval;
  if (nchal) {
    std::vector<HostFr> acc;
    const HostFr x = HostFr::from_limbs(sp->public_x);
    HostFr pw = HostFr::one();
    for (size_t j = 0; j < nchal; j++) {
      size_t at = cidx.size();
      for (size_t q = 0; q < cidx.size(); q++)
        if (cidx[q] == st->offsets[j]) at = q;
      if (at == cidx.size()) {
        cidx.push_back(st->offsets[j]);
        acc.push_back(HostFr::zero());
      }
      acc[at] = HostFr::add(acc[at], pw);
      pw = HostFr::mul(pw, x);
    }
    cval.resize(4 * acc.size());
    for (size_t q = 0; q < acc.size(); q++) memcpy(&cval[4 * q], acc[q].l, 32);
  }
  Scratch s_sc;
  if (nchal) {
    if ((rc = s_sc.alloc(8 * cidx.size() + 32 * cval.size() / 4, s))) return rc;
    uint64_t* d_idx = static_cast<uint64_t*>(s_sc.ptr);
    uint64_t* d_val = d_idx + cidx.size();
    PK_CUDA(cudaMemcpyAsync(d_idx, cidx.data(), 8 * cidx.size(), cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaMemcpyAsync(d_val, cval.data(), 8 * cval.size(), cudaMemcpyHostToDevice, s));
    const unsigned blocks = (unsigned)std::min<size_t>((cidx.size() + 255) / 256, 1024);
    scatter_fr_kernel<<<blocks, 256, 0, s>>>(st2 + 4 * 3 * n, d_idx, d_val, cidx.size());
    PK_CHECK_LAUNCH("scatter_fr_kernel");
  }
  const bool cached = r1cs->row_ptr_t[0] && r1cs->row_ptr_t[1] && r1cs->row_ptr_t[2];
  FusedSlots fs;
  if ((rc = fused_slots(&fs))) return rc;
  for (int k = 0; k < 3; k++) {
    Scratch s_t;
    const uint64_t* rp_t = r1cs->row_ptr_t[k];
    const uint32_t* cl_t = r1cs->cols_t[k];
    const uint64_t* vl_t = r1cs->vals_t[k];
    const size_t nnz = r1cs->nnz[k];
    if (!cached) {
      const size_t rp_bytes = round256(8 * (nw + 1)), cl_bytes = round256(4 * (nnz ? nnz : 1));
      if ((rc = s_t.alloc(rp_bytes + cl_bytes + 32 * (nnz ? nnz : 1), s))) return rc;
      uint8_t* b = static_cast<uint8_t*>(s_t.ptr);
      uint64_t* rp = reinterpret_cast<uint64_t*>(b);
      uint32_t* cl = reinterpret_cast<uint32_t*>(b + rp_bytes);
      uint64_t* vl = reinterpret_cast<uint64_t*>(b + rp_bytes + cl_bytes);
      if ((rc = pkg_csr_transpose(r1cs->row_ptr[k], r1cs->cols[k], r1cs->vals[k], nc, nw, nnz, rp,
                                  cl, vl, reinterpret_cast<pkg_stream_t>(s))))
        return rc;
      rp_t = rp;
      cl_t = cl;
      vl_t = vl;
    } else {
      PK_REQUIRE(cl_t && vl_t, "transpose %d of the R1CS is incomplete", k);
    }
    if ((rc = spmv_device(rp_t, cl_t, vl_t, nw, nc, eq, alph, err, s, nnz))) return rc;
    uint64_t* a1 = st1 + 4 * n * (base + (size_t)k);
    uint64_t* a2 = st2 + 4 * n * (size_t)k;
    PK_CUDA(cudaMemcpyAsync(a1, alph, 32 * w1_size, cudaMemcpyDeviceToDevice, s));
    if (w2_size)
      PK_CUDA(cudaMemcpyAsync(a2, alph + 4 * w1_size, 32 * w2_size, cudaMemcpyDeviceToDevice, s));
    // compute_alpha_evals (prefix_covector.rs:212-223) on each part
    if ((rc = dot_device(a1, st->poly[0], w1_size, fs.dev + 4 * k, part, s, fs.ticket))) return rc;
    if ((rc = dot_device(a2, st->poly[1], w2_size, fs.dev + 4 * (3 + k), part, s, fs.ticket)))
      return rc;
  }
  if (nchal &&  // compute_challenge_eval (prefix_covector.rs:326-338) on w2
      (rc = dot_device(st2 + 4 * 3 * n, st->poly[1], n, fs.dev + 4 * 6, part, s, fs.ticket)))
    return rc;
  uint64_t sums[7][4];
  if ((rc = fused_read(sums, fs, 32 * (nchal ? 7 : 6), s))) return rc;
  memcpy(sp->evals, sums, 96);
  memcpy(out->evals2, sums[3], 96);
  if (nchal) memcpy(out->challenge_eval, sums[6], 32);
  uint32_t h_err2 = 0;  // the transposed products' column check
  if ((rc = read_small(&h_err2, err, 4, s))) return rc;
  PK_REQUIRE(!h_err2, "R1CS column index out of range");
  // the messages in the reference's order (:328-348)
  for (int k = 0; k < 3; k++) pkg_transcript_absorb(&st->t, sp->evals[k]);
  for (int k = 0; k < 3; k++) pkg_transcript_absorb(&st->t, out->evals2[k]);
  std::vector<uint64_t> xpow(4 * (np + 1));
  if (np) {  // compute_public_eval on w1 (prefix_covector.rs:226-240)
    public_weight_host(pubw.data(), np, sp->public_x, xpow.data(), sp->public_eval);
    pkg_transcript_absorb(&st->t, sp->public_eval);
  }
  if (nchal) pkg_transcript_absorb(&st->t, out->challenge_eval);
  sp->transcript = st->t;

  // w1's statements: the public weight first (:350-356), the blinding
  // covector last (OffsetCovector at w1_size); then both WHIR proofs on one
  // transcript, each computing its statements' values from its polynomials
  if (np) PK_CUDA(cudaMemcpyAsync(st1, xpow.data(), 32 * (np + 1), cudaMemcpyHostToDevice, s));
  std::vector<uint64_t> bw(16 * m0);
  blinding_weights_host(&sp->alpha[0][0], m0, bw.data());
  PK_CUDA(cudaMemcpyAsync(st1 + 4 * n * (base + 3) + 4 * w1_size, bw.data(), 32 * 4 * m0,
                          cudaMemcpyHostToDevice, s));
  pkg_transcript tw = st->t;
  if ((rc = whir_prove_device(&st->whir, &tw, st->poly[0], st->cw[0], st->layers[0], st->ood[0],
                              st1, ncov1, nullptr, nullptr, whir_proof1, s)))
    return rc;
  return whir_prove_device(&st->whir, &tw, st->poly[1], st->cw[1], st->layers[1], st->ood[1], st2,
                           ncov2, nullptr, nullptr, whir_proof2, s);
}
