// prove.cu -- pkg_spartan_prove: the Spartan prover's work up to WHIR's own
// prove rounds, device-resident from the witness to the covector
// evaluations (provekit/prover/src/whir_r1cs.rs:82-301,
// provekit/r1cs-compiler/src/whir_r1cs.rs:48-92); pkg_prove_r1cs: the same
// with whir's commitment OOD samples and the WHIR proof (pkg_whir_prove) of
// the statements' evaluations, a whole proof.
//
// Device data: the padded witness polynomial (2^m Fr), its RS codeword and
// Merkle layers, the a/b/c sumcheck tables (2^m0 Fr each), eq(alpha), the
// transposed matrices and the alpha covectors.  The host keeps the
// transcript and reads back only the root, three Fr per sumcheck round and
// the final scalars.
#include <chrono>
#include <cstring>
#include <vector>

#include "fr_host.hpp"
#include "internal.cuh"
#include "pk_common.cuh"
#include "rs_internal.cuh"
#include "sky_host.hpp"

namespace pk {

static size_t ceil_log2(size_t n) {  // utils::next_power_of_two (utils/mod.rs:71-79)
  size_t p = 1, k = 0;
  while (p < n) {
    p <<= 1;
    k++;
  }
  return k;
}

// Host wall-clock of the calling thread's last pkg_spartan_prove, per stage;
// every stage but the witness bounds (only enqueued; their device time falls
// in the zk sumcheck's) ends with a synchronisation, so these are the
// stages' device time plus their host work.
thread_local double g_stage_ms[PKG_PROVE_STAGES];

struct StageClock {
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(int k) {
    const auto now = std::chrono::steady_clock::now();
    g_stage_ms[k] = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
  }
};

int public_challenge(const uint64_t* witness, size_t np, uint64_t* pubw, pkg_transcript* t,
                     uint64_t hash[4], uint64_t x[4], cudaStream_t s) {
  memset(hash, 0, 32);
  if (np) {
    int rc = read_small(pubw, witness, 32 * (np + 1), s);
    if (rc) return rc;
    auto w = [pubw](size_t i) { return HostFr::from_mont(HostFr::from_limbs(pubw + 4 * i)); };
    HostFr h = HostSky::compress(w(1), np > 1 ? w(2) : HostFr::zero());
    for (size_t i = 3; i <= np; i++) h = HostSky::compress(h, w(i));
    memcpy(hash, h.l, 32);
  }
  const HostFr hm = HostFr::to_mont(HostFr::from_limbs(hash));
  pkg_transcript_absorb(t, hm.l);
  return pkg_transcript_squeeze(t, x);
}

void public_weight_host(const uint64_t* pubw, size_t np, const uint64_t x_words[4], uint64_t* xpow,
                        uint64_t eval[4]) {
  const HostFr x = HostFr::from_limbs(x_words);
  HostFr pw = HostFr::one(), acc = HostFr::zero();
  for (size_t i = 0; i <= np; i++) {
    memcpy(xpow + 4 * i, pw.l, 32);
    acc = HostFr::add(acc, HostFr::mul(pw, HostFr::from_limbs(pubw + 4 * i)));
    pw = HostFr::mul(pw, x);
  }
  memcpy(eval, acc.l, 32);
}

void blinding_weights_host(const uint64_t* alpha, size_t m0, uint64_t* bw) {
  for (size_t i = 0; i < m0; i++) {
    HostFr pw = HostFr::one();
    const HostFr a = HostFr::from_limbs(alpha + 4 * i);
    for (int k = 0; k < 4; k++) {
      memcpy(bw + 4 * (4 * i + k), pw.l, 32);
      pw = HostFr::mul(pw, a);
    }
  }
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_last_prove_stages(double ms[PKG_PROVE_STAGES]) {
  PK_REQUIRE(ms, "null output");
  memcpy(ms, g_stage_ms, sizeof g_stage_ms);
  return PKG_OK;
}

extern "C" int pkg_r1cs_sizing(size_t num_constraints, size_t num_witnesses, size_t* m_out,
                               size_t* m0_out) {
  PK_REQUIRE(m_out && m0_out, "null output");
  PK_REQUIRE(num_constraints >= 1 && num_witnesses >= 1, "empty R1CS");
  size_t m = ceil_log2(num_witnesses), m0 = ceil_log2(num_constraints);
  if (m < 13) m = 13;  // MIN_WHIR_NUM_VARIABLES
  if (m0 < 1) m0 = 1;  // MIN_SUMCHECK_NUM_VARIABLES
  if ((size_t(1) << m) - num_witnesses < 4 * m0) m++;
  *m_out = m;
  *m0_out = m0;
  return PKG_OK;
}

// With whir == nullptr the commitment's root alone enters the transcript and
// the proof ends at the covector evaluations (pkg_spartan_prove); with whir,
// the commitment's OOD samples follow the root and the WHIR proof of the
// statements ends it (pkg_prove_r1cs): the public weight when there are
// public inputs, the three zero-padded covectors and the blinding covector.
static int spartan_prove_impl(const pkg_r1cs* r1cs, const uint64_t* witness,
                              uint64_t blinding_seed, uint64_t transcript_domain, unsigned ff,
                              unsigned lr, pkg_spartan_proof* out, const pkg_whir_params* whir,
                              uint64_t* whir_commit_words, uint64_t* whir_proof,
                              pkg_stream_t stream) {
  PK_REQUIRE(r1cs && witness && out, "null pointer");
  PK_REQUIRE(aligned16(witness), "witness must be 16-byte aligned");
  const size_t nc = r1cs->num_constraints, nw = r1cs->num_witnesses, w1_size = nw;
  size_t m = 0, m0 = 0;
  int rc = pkg_r1cs_sizing(nc, nw, &m, &m0);
  if (rc) return rc;
  PK_REQUIRE(m0 <= 30 && m <= 28 && ff <= m && lr <= 8, "instance too large (m=%zu, m0=%zu)", m,
             m0);
  PK_REQUIRE(r1cs->num_public_inputs + 1 <= nw, "%zu public inputs but %zu witnesses",
             r1cs->num_public_inputs, nw);
  if (whir) {
    PK_REQUIRE(whir_commit_words && whir_proof, "null WHIR output");
    PK_REQUIRE(pkg_whir_proof_words(whir, 3) != 0, "invalid WHIR parameters");
    PK_REQUIRE(whir->num_variables == m, "WHIR parameters for %u variables, the R1CS needs %zu",
               whir->num_variables, m);
    PK_REQUIRE(whir->batch_size == 1 || whir->batch_size == 2,
               "WHIR batch of %u: the witness is committed alone or with one blinding "
               "polynomial", whir->batch_size);
  }
  memset(out, 0, sizeof *out);
  memset(g_stage_ms, 0, sizeof g_stage_ms);
  StageClock clk;
  out->m = m;
  out->m0 = m0;
  cudaStream_t s = as_stream(stream);
  const uint64_t dom[4] = {transcript_domain, 0, 0, 0};
  rc = pkg_transcript_init(&out->transcript, dom);
  if (rc) return rc;

  // ---- commit (whir_r1cs.rs:82-140)
  const size_t n = size_t(1) << m, M = size_t(1) << ff, L = n >> ff, cw_len = L << lr;
  const size_t n0 = size_t(1) << m0;
  // whir-ZK (a WHIR batch of 2): the witness polynomial is committed with a
  // random blinding polynomial g of the same length in one tree
  const unsigned nb = whir ? whir->batch_size : 1;
  Scratch s_poly, s_cw, s_layers, s_tab, s_misc;
  if ((rc = s_poly.alloc(32 * n * nb, s))) return rc;
  if ((rc = s_cw.alloc(32 * M * nb * cw_len, s))) return rc;
  if ((rc = s_layers.alloc(32 * (2 * cw_len - 1), s))) return rc;
  if ((rc = s_tab.alloc(32 * 3 * n0, s))) return rc;
  uint64_t* poly = static_cast<uint64_t*>(s_poly.ptr);
  uint64_t* cw = static_cast<uint64_t*>(s_cw.ptr);
  uint8_t* layers = static_cast<uint8_t*>(s_layers.ptr);
  uint64_t* ta = static_cast<uint64_t*>(s_tab.ptr);
  uint64_t* tb = ta + 4 * n0;
  uint64_t* tc = tb + 4 * n0;
  std::vector<uint64_t> g(16 * m0);
  pkg_sample_fr(blinding_seed, 4 * m0, g.data(), 1);  // generate_blinding_univariates, seeded
  PK_CUDA(cudaMemcpyAsync(poly, witness, 32 * nw, cudaMemcpyDeviceToDevice, s));
  PK_CUDA(cudaMemsetAsync(poly + 4 * nw, 0, 32 * (n - nw), s));
  PK_CUDA(cudaMemcpyAsync(poly + 4 * w1_size, g.data(), 32 * 4 * m0, cudaMemcpyHostToDevice, s));
  uint64_t* mask = poly + 4 * n;  // the blinding polynomial (batch of 2)
  if (nb == 2 && (rc = pkg_sample_fr_indexed(blinding_seed ^ kMaskSeed, 0, n, mask, stream)))
    return rc;
  if ((rc = rs_encode_device(poly, M * nb, L, nullptr, 0, cw_len, cw, s))) return rc;
  if ((rc = merkle_tree_fr_device(cw, M * nb, cw_len, PKG_LEAF_CANONICAL, layers, s))) return rc;
  uint64_t ood_points[4 * 5];
  if (whir) {
    // whir's commit: the root (read there, its words are the commitment's
    // first four), then the OOD samples of the committed polynomial
    if ((rc = pkg_whir_commit_ood(whir, &out->transcript, poly, layers, whir_commit_words,
                                  ood_points, stream)))
      return rc;
    memcpy(out->root, whir_commit_words, 32);
  } else {
    if ((rc = read_small(out->root, layers + 32 * (2 * cw_len - 2), 32, s))) return rc;
    HostFr root = HostFr::to_mont(HostFr::from_limbs(reinterpret_cast<const uint64_t*>(out->root)));
    pkg_transcript_absorb(&out->transcript, root.l);
  }
  clk.mark(0);

  // ---- witness bounds (sumcheck.rs:163-179)
  // partial sums of dot_device (<= 4 * SMs CTAs); its results go to the
  // thread's fused slots
  const size_t nparts = 4 * (size_t)sm_count();
  if ((rc = s_misc.alloc(256 + 32 * nparts, s))) return rc;
  uint32_t* err = static_cast<uint32_t*>(s_misc.ptr);
  uint64_t* part = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(s_misc.ptr) + 256);
  PK_CUDA(cudaMemsetAsync(err, 0, 4, s));
  // a = A w, b = B w, c = a o b, zero-padded to 2^m0: one launch
  if ((rc = witness_bounds_device(r1cs, witness, n0, ta, tb, tc, err, s))) return rc;

  // The witness bounds' error flag goes to a spare word of the thread's
  // mapped slots without a synchronisation; the sumcheck's first round
  // trip, which follows the copy in the stream, makes it readable.  The host
  // meanwhile starts the sumcheck (its challenges, the eq table), so the
  // device is not left idle for a read here.
  volatile uint32_t* h_err = nullptr;
  if ((rc = fused_aux_word(const_cast<uint32_t**>(&h_err)))) return rc;
  *h_err = 0;
  PK_CUDA(cudaMemcpyAsync(const_cast<uint32_t*>(h_err), err, 4, cudaMemcpyDeviceToHost, s));
  clk.mark(1);

  // ---- zk sumcheck (whir_r1cs.rs:519-621); the blinding coefficients in
  // w1[offset .. offset + 4 m0] are g, written above
  rc = pkg_spartan_sumcheck(ta, tb, tc, m0, g.data(), g.data(), &out->transcript, &out->r[0][0],
                            out->rho, out->sum_g, &out->coeffs[0][0], &out->alpha[0][0],
                            out->blinding_eval, stream);
  if (rc) {
    cudaStreamSynchronize(s);  // the flag's copy must not land in a later proof's word
    return rc;
  }
  PK_REQUIRE(!*h_err, "R1CS column index out of range");
  clk.mark(2);
  FusedSlots fs;  // the dots below write their results to the thread's slots
  if ((rc = fused_slots(&fs))) return rc;

  // ---- eq(alpha) and the transposed products (sumcheck.rs:195-227)
  // The covectors: one nw-entry buffer, or for the WHIR proof the
  // statements of prove_from_alphas (whir_r1cs.rs:258-301), each 2^m entries:
  // [public weight?, A^T eq, B^T eq, C^T eq, blinding covector].
  const size_t np = r1cs->num_public_inputs;
  const size_t sbase = np ? 1 : 0, nstm = sbase + 4;
  Scratch s_eq, s_alph;
  if ((rc = s_eq.alloc(32 * nc, s))) return rc;
  if ((rc = s_alph.alloc(32 * (whir ? nstm * n : nw), s))) return rc;
  uint64_t* eq = static_cast<uint64_t*>(s_eq.ptr);
  uint64_t* cov = static_cast<uint64_t*>(s_alph.ptr);
  if (whir) PK_CUDA(cudaMemsetAsync(cov, 0, 32 * nstm * n, s));
  // out->alpha stays valid and unchanged until the evaluations' read below
  if ((rc = eq_hypercube_device(&out->alpha[0][0], m0, nc, eq, s, false))) return rc;
  // public weights: the public inputs' hash into the transcript, then x
  std::vector<uint64_t> pubw(4 * (np + 1));  // w[0 ..= np], Montgomery form
  if ((rc = public_challenge(witness, np, pubw.data(), &out->transcript, out->public_hash,
                             out->public_x, s)))
    return rc;
  clk.mark(3);
  // the transposes: the resident circuit's (built once), else built here
  const bool cached = r1cs->row_ptr_t[0] && r1cs->row_ptr_t[1] && r1cs->row_ptr_t[2];
  for (int k = 0; k < 3; k++) {
    uint64_t* alph = whir ? cov + 4 * n * (sbase + (size_t)k) : cov;
    Scratch s_t;
    const uint64_t* rp_t = r1cs->row_ptr_t[k];
    const uint32_t* cl_t = r1cs->cols_t[k];
    const uint64_t* vl_t = r1cs->vals_t[k];
    if (!cached) {
      const size_t nnz = r1cs->nnz[k];
      const size_t rp_bytes = ((8 * (nw + 1) + 255) / 256) * 256;
      const size_t cl_bytes = ((4 * (nnz ? nnz : 1) + 255) / 256) * 256;
      if ((rc = s_t.alloc(rp_bytes + cl_bytes + 32 * (nnz ? nnz : 1), s))) return rc;
      uint8_t* base = static_cast<uint8_t*>(s_t.ptr);
      uint64_t* rp = reinterpret_cast<uint64_t*>(base);
      uint32_t* cl = reinterpret_cast<uint32_t*>(base + rp_bytes);
      uint64_t* vl = reinterpret_cast<uint64_t*>(base + rp_bytes + cl_bytes);
      rc = pkg_csr_transpose(r1cs->row_ptr[k], r1cs->cols[k], r1cs->vals[k], nc, nw, nnz, rp, cl,
                             vl, stream);
      if (rc) return rc;
      rp_t = rp;
      cl_t = cl;
      vl_t = vl;
    } else {
      PK_REQUIRE(cl_t && vl_t, "transpose %d of the R1CS is incomplete", k);
    }
    if ((rc = spmv_device(rp_t, cl_t, vl_t, nw, nc, eq, alph, err, s, r1cs->nnz[k]))) return rc;
    // create_weights_and_evaluations (:623-642): the zero padding adds nothing
    if ((rc = dot_device(alph, poly, nw, fs.dev + 4 * k, part, s, fs.ticket))) return rc;
  }
  // the three evaluations read back at once, then absorbed in order
  if ((rc = fused_read(&out->evals[0][0], fs, 96, s))) return rc;
  for (int k = 0; k < 3; k++) pkg_transcript_absorb(&out->transcript, out->evals[k]);
  // the public weight's evaluation <[1, x, .., x^np], w> and its message
  // (compute_public_weight_evaluation, :654-663, :275-282)
  std::vector<uint64_t> xpow(4 * (np + 1));
  if (np) {
    public_weight_host(pubw.data(), np, out->public_x, xpow.data(), out->public_eval);
    pkg_transcript_absorb(&out->transcript, out->public_eval);
  }
  clk.mark(4);
  if (whir) {
    // the public weight and the blinding covector expand_powers::<4>(alpha)
    // at the blinding offset (OffsetCovector, prefix_covector.rs:90-112)
    if (np)
      PK_CUDA(cudaMemcpyAsync(cov, xpow.data(), 32 * (np + 1), cudaMemcpyHostToDevice, s));
    std::vector<uint64_t> bw(16 * m0);
    blinding_weights_host(&out->alpha[0][0], m0, bw.data());
    PK_CUDA(cudaMemcpyAsync(cov + 4 * n * (sbase + 3) + 4 * w1_size, bw.data(), 32 * 4 * m0,
                            cudaMemcpyHostToDevice, s));
    // statement values of w: [public_eval?, evals, blinding_eval]; for
    // whir-ZK also every statement's value on the blinding polynomial g
    std::vector<uint64_t> vals(4 * nstm * nb);
    size_t at = 0;
    if (np) {
      memcpy(vals.data(), out->public_eval, 32);
      at = 4;
    }
    memcpy(vals.data() + at, &out->evals[0][0], 96);
    memcpy(vals.data() + at + 12, out->blinding_eval, 32);
    for (size_t k = 0; nb == 2 && k < nstm; k++)
      if ((rc = dot_device(cov + 4 * n * k, mask, n, fs.dev + 4 * k, part, s, fs.ticket)))
        return rc;
    if (nb == 2 && (rc = fused_read(vals.data() + 4 * nstm, fs, 32 * nstm, s))) return rc;
    // host sources above are pageable: staged before the copies returned
    pkg_transcript tw = out->transcript;
    if ((rc = whir_prove_device(whir, &tw, poly, cw, layers, ood_points, cov, nstm, vals.data(),
                                nullptr, whir_proof, s)))
      return rc;
    clk.mark(5);
  }
  return PKG_OK;
}

extern "C" int pkg_spartan_prove(const pkg_r1cs* r1cs, const uint64_t* witness,
                                 uint64_t blinding_seed, uint64_t transcript_domain,
                                 unsigned ff, unsigned lr, pkg_spartan_proof* out,
                                 pkg_stream_t stream) {
  return spartan_prove_impl(r1cs, witness, blinding_seed, transcript_domain, ff, lr, out, nullptr,
                            nullptr, nullptr, stream);
}

extern "C" int pkg_prove_r1cs(const pkg_r1cs* r1cs, const uint64_t* witness,
                              uint64_t blinding_seed, uint64_t transcript_domain,
                              const pkg_whir_params* whir, pkg_spartan_proof* out,
                              uint64_t* whir_commit_words, uint64_t* whir_proof,
                              pkg_stream_t stream) {
  PK_REQUIRE(whir, "null WHIR parameters");
  return spartan_prove_impl(r1cs, witness, blinding_seed, transcript_domain, whir->folding_factor,
                            whir->log_inv_rate, out, whir, whir_commit_words, whir_proof, stream);
}
