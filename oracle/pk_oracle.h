/*
 * pk_oracle.h -- CPU restatement of ProveKit's Spartan+WHIR prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle for the CUDA
 * implementation in provekit_b200/.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference arm may load it, and only as a checker
 * or as the timed CPU baseline -- never as a fallback for the product path.
 *
 * Field elements are BN254 Fr, 4 x u64 little-endian limbs.  "mont" means the
 * arkworks in-memory form x*2^256 mod p, always fully reduced; "canonical"
 * means x itself in [0, p).
 *
 * Parity pins: Skyscraper KATs (skyscraper/core/src/reference.rs:104-188),
 * sumcheck helper KATs (provekit/common/src/utils/sumcheck.rs:229-436),
 * Poseidon2 KATs (poseidon2/src/permutation.rs:182-195, hash.rs:53-70).
 * The NTT root of unity is derived as arkworks does (generator 5, two-adicity
 * 28); no reference golden output pins NTT bytes directly.
 */
#ifndef PK_ORACLE_H
#define PK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- field ---------------------------------------------------------- */
void pko_fr_mul(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]);
void pko_fr_add(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]);
void pko_fr_sub(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]);
void pko_fr_to_mont(uint64_t r[4], const uint64_t a[4]);   /* a canonical */
void pko_fr_from_mont(uint64_t r[4], const uint64_t a[4]);
void pko_fr_inv(uint64_t r[4], const uint64_t a[4]);         /* mont in/out */
void pko_fr_root_of_unity(uint64_t r[4], uint64_t n);        /* mont out    */
void pko_to_mont_many(uint64_t *v, size_t n);
void pko_from_mont_many(uint64_t *v, size_t n);

/* Seeded ChaCha20 Fr sampler (RFC 8439 block function, 64-bit counter,
 * key = seed LE in the first 8 bytes).  254-bit mask + rejection; output in
 * Montgomery form when mont != 0. */
void pko_sample_fr(uint64_t seed, size_t n, uint64_t *out, int mont);
/* Indexed sampler (no rejection, any element computable alone): out[i] =
 * lo + hi 2^253 mod p (Montgomery form), lo and hi the two 32-byte halves of
 * ChaCha20 block start + i (key = seed LE, nonce word 1), each read as a
 * little-endian integer masked to 253 bits. */
void pko_sample_fr_indexed(uint64_t seed, uint64_t start, size_t n, uint64_t *out);

/* ---- ntt crate (ntt/src/ntt.rs) --------------------------------------- */
int  pko_ntt_nr(uint64_t *values, size_t len, size_t codeword_size, size_t num_groups);
int  pko_intt_rn(uint64_t *values, size_t len);
void pko_roots_reverse_ordered(uint64_t *out, size_t order);   /* order/2 entries */

/* ---- RSFr::interleaved_encode (provekit/common/src/ntt.rs:51-100) ------ */
/* messages: num_messages x message_length, message-major. */
int pko_rs_interleaved_encode(const uint64_t *messages, size_t num_messages,
                              size_t message_length, const uint64_t *masks,
                              size_t mask_len, size_t codeword_length,
                              uint64_t *out);
void pko_rs_evaluation_points(size_t codeword_length, const size_t *indices,
                              size_t n, uint64_t *out);

/* ---- Skyscraper (skyscraper/core/src) ---------------------------------- */
void pko_sky_compress(uint64_t out[4], const uint64_t l[4], const uint64_t r[4]);
int  pko_sky_compress_many(const uint8_t *messages, size_t n, uint8_t *hashes);
void pko_sky_permute(uint64_t l[4], uint64_t r[4]);               /* canonical */
void pko_sky_ss(int round, uint64_t l[4], uint64_t r[4]);
void pko_sky_bb(int round, uint64_t l[4], uint64_t r[4]);
uint8_t pko_sky_sbox(uint8_t v);
int  pko_hash_many(size_t size, const uint8_t *input, size_t count, uint8_t *output);
/* Merkle tree over count leaves of leaf_size bytes: writes 2*count-1
 * digests, level by level (leaf digests first, root last). */
int  pko_merkle_tree(const uint8_t *leaves, size_t leaf_size, size_t count,
                     uint8_t *layers);
/* PoW: smallest nonce with compress(challenge, [nonce,0,0,0]) < threshold. */
uint64_t pko_sky_pow_solve(const uint64_t challenge[4], const uint64_t threshold[4]);

/* ---- Spartan sumcheck (provekit/common/src/utils/sumcheck.rs) ---------- */
void pko_calculate_eq(uint64_t out[4], const uint64_t *r, const uint64_t *alpha, size_t n);
int  pko_eq_hypercube(const uint64_t *r, size_t nr, size_t num_entries, uint64_t *out);
/* One round of the Spartan map-reduce over tables a,b,c,eq of length size;
 * fold != NULL applies the quarter-layout fold first (tables halve). */
int  pko_spartan_round(uint64_t *a, uint64_t *b, uint64_t *c, uint64_t *eq,
                       size_t size, const uint64_t *fold, uint64_t out[12]);
/* CSR SpMV: y[row] = sum_k vals[k] * x[cols[k]] over row_ptr[row]..row_ptr[row+1]. */
int  pko_spmv(const uint64_t *row_ptr, const uint32_t *cols, const uint64_t *vals,
              size_t num_rows, const uint64_t *x, uint64_t *y);
void pko_eval_cubic(uint64_t out[4], const uint64_t poly[16], const uint64_t x[4]);
void pko_blinding_coeffs(const uint64_t *g, size_t n, size_t compute_for,
                         const uint64_t *alphas, uint64_t out[16]);
void pko_dot(uint64_t out[4], const uint64_t *a, const uint64_t *b, size_t n);

/* ---- Fiat-Shamir transcript stand-in ------------------------------------ */
/* The reference's transcript is spongefish's DuplexSponge over
 * skyscraper::reference::permute (provekit/common/src/skyscraper/sponge.rs:27-41);
 * spongefish is not available, so its byte layout is replaced by this
 * minimal duplex: state (l, r) canonical; init: l = domain mod p, r = 0,
 * permute; absorb(x): l += canonical(x), permute; squeeze: permute, return l
 * (Montgomery form out). */
typedef struct { uint64_t l[4], r[4]; } pko_transcript;
void pko_transcript_init(pko_transcript *t, const uint64_t domain[4]);
void pko_transcript_absorb(pko_transcript *t, const uint64_t x_mont[4]);
void pko_transcript_squeeze(pko_transcript *t, uint64_t out_mont[4]);

/* run_zk_sumcheck_prover (provekit/prover/src/whir_r1cs.rs:519-621) over
 * tables a, b, c of length 2^m0 (already padded; modified in place), the
 * blinding polynomial g (m0 x 4 Fr) and the w1 polynomial (blinding
 * coefficients at blinding_offset).  Outputs: r (m0), rho, sum_g, the 4*m0
 * round coefficients, alpha (m0), blinding_eval. */
int pko_spartan_sumcheck(pko_transcript *t, uint64_t *a, uint64_t *b, uint64_t *c, size_t m0,
                         const uint64_t *g, const uint64_t *w1, size_t blinding_offset,
                         uint64_t *r_out, uint64_t rho_out[4], uint64_t sum_g_out[4],
                         uint64_t *coeffs_out, uint64_t *alpha_out, uint64_t blinding_eval[4]);

/* Spartan prove core (the prover's work before WHIR's own rounds):
 * WhirR1CSScheme::new_for_r1cs sizing (provekit/r1cs-compiler/src/whir_r1cs.rs:48-92),
 * commit (provekit/prover/src/whir_r1cs.rs:82-140) with the blinding
 * polynomial drawn from the ChaCha sampler (seed) instead of thread_rng and
 * the commitment = RS encode + Skyscraper tree of 2^ff contiguous messages,
 * prove_noir (:143-187) up to the WHIR prove call: witness bounds, zk
 * sumcheck, eq(alpha), transposed SpMV, public-weight challenge, the three
 * covector evaluations (:247-301). */
typedef struct {
    size_t num_constraints, num_witnesses;
    const uint64_t *row_ptr[3];   /* A, B, C: num_constraints + 1 */
    const uint32_t *cols[3];
    const uint64_t *vals[3];
    size_t num_public_inputs;     /* the public inputs are witness[1 ..= this] */
} pko_r1cs;
typedef struct {
    size_t m, m0;
    uint8_t root[32];
    uint64_t r[30][4], coeffs[120][4], alpha[30][4];
    uint64_t rho[4], sum_g[4], blinding_eval[4], public_x[4], evals[3][4];
    pko_transcript transcript;
    uint64_t public_hash[4], public_eval[4]; /* canonical hash; mont eval (0 without publics) */
} pko_spartan_proof;
int pko_spartan_prove(const pko_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                      uint64_t domain, unsigned folding_factor, unsigned log_inv_rate,
                      pko_spartan_proof *out);

/* ---- Poseidon2 t = 4 (poseidon2/src) ----------------------------------- */
void pko_poseidon2_permutation(uint64_t state[16]);                      /* mont in/out */
void pko_poseidon2_hash(uint64_t out[4], const uint64_t *inputs, size_t n); /* mont */

/* ---- WHIR prove-round building blocks ----------------------------------
 * Arithmetic conventions follow the reference's WHIR verifier restated in Go
 * (recursive-verifier/app/...): MultivarPoly (utilities/utilities.go:16-23),
 * UnivarPoly (:25-39), ExpandFromUnivariate (:183-191),
 * EvaluateQuadraticPolynomialFromEvaluationList (:149-155),
 * verifyMerkleTreeProofs and getStirChallenges (circuit/whir_utilities.go:14-79).
 * Field values are Montgomery form unless stated. */
/* w_j = prod_t alpha[t]^(bit t of j), j < 2^k: the coefficient of row entry j
 * in MultivarPoly(row, alpha). */
void pko_multilinear_weights(uint64_t *w, const uint64_t *alpha, unsigned k);
/* out[i] = sum_j w_j * coeffs[j*(n>>k) + i], i < n >> k: the folded polynomial
 * whose RS codeword is the fold of the interleaved codeword's rows. */
int  pko_whir_fold_coeffs(const uint64_t *coeffs, size_t n, unsigned k, const uint64_t *alpha,
                          uint64_t *out);
/* out[i] = MultivarPoly(rows[i*2^k .. (i+1)*2^k), alpha) (computeFold). */
int  pko_whir_fold_rows(const uint64_t *rows, size_t nrows, unsigned k, const uint64_t *alpha,
                        uint64_t *out);
/* sum_i coeffs[i] * z^i (UnivarPoly, Horner). */
void pko_poly_eval(uint64_t out[4], const uint64_t *coeffs, size_t n, const uint64_t z[4]);
/* out[n-1-i] = z^(2^i) (ExpandFromUnivariate). */
void pko_expand_from_univariate(uint64_t *out, const uint64_t z[4], size_t n);
/* Authentication path of leaf idx in a layers array (leaves first, root
 * last): path[l] = node (idx >> l) ^ 1 of level l, l < log2(num_leaves). */
int  pko_merkle_open(const uint8_t *layers, size_t num_leaves, uint64_t idx, uint8_t *path);
/* verifyMerkleTreeProofs for one leaf: leaf hash = left fold of compress over
 * the leaf's field elements (canonical limbs), then up the path with the
 * index bits choosing sides.  Returns 1 when the root matches. */
int  pko_merkle_verify(const uint64_t *leaf_canonical, size_t fr_per_leaf, uint64_t idx,
                       const uint8_t *path, size_t depth, const uint8_t root[32]);
/* getStirChallenges: ceil(log2(folded)/8) big-endian challenge bytes per
 * query, reduced to the low log2(folded) bits. */
void pko_stir_indices(const uint8_t *bytes, size_t folded_domain_size, size_t nq, uint64_t *out);
/* WHIR sumcheck round over tables f, w (size entries, top variable first):
 * with fold, first t[i] += fold*(t[i+size/2]-t[i]) for i < size/2 and the
 * live size halves; then out = (h(0), h(1), h(2)) of
 * h(X) = sum_b f(X, b) w(X, b) over the live tables' top variable. */
int  pko_whir_sumcheck_round(uint64_t *f, uint64_t *w, size_t size, const uint64_t *fold,
                             uint64_t out[12]);
/* w[b] += sum_j coeffs[j] * eq(points[j], b) for b < 2^nv, point
 * coordinate 0 on the top bit of b (as pko_eq_hypercube). */
int  pko_eq_accumulate(uint64_t *w, size_t nv, const uint64_t *points, const uint64_t *coeffs,
                       size_t npts);

/* ---- WHIR round orchestration (pk_oracle_whir.c) --------------------------
 * A whole WHIR proof of linear statements <a_k, c> = v_k about a committed
 * coefficient vector c (2^n Fr), in the round order of the reference's Go
 * verifier runWhir (recursive-verifier/app/circuit/whir.go:587-724), with
 *  - query points from RSFr::evaluation_points (provekit/common/src/ntt.rs:22-42:
 *    row i of a codeword of L rows sits at w_L^bitrev(i));
 *  - 2^k contiguous messages per codeword row (pko_whir_fold_coeffs), so a
 *    sumcheck binds the top bit of the coefficient index first and the
 *    round's fold randomness is the reverse of its sumcheck challenges;
 *  - the sumcheck over f^(b) * w(b) on the hypercube, f^ = zeta(c) (subset
 *    sums), linear statements as w = mobius^T(a) (superset differences);
 *  - the transcript stand-in above; PoW = pko_sky_pow_solve with threshold
 *    floor(p / 2^bits) (CheckPoW, utilities/utilities.go:104-139).
 * whir's own byte layout and schedule are un-vendored; this is the protocol
 * the device prover must reproduce word for word. */
#define PKO_WHIR_MAX_ROUNDS 16
typedef struct {
    uint32_t num_variables;   /* n: the committed vector has 2^n entries      */
    uint32_t folding_factor;  /* k, 1..6 (constant over the rounds)            */
    uint32_t log_inv_rate;    /* starting rate 2^-log_inv_rate                */
    uint32_t num_rounds;      /* R: rounds with a new commitment              */
    uint32_t final_vars;      /* n - (R+1) k: variables sent in the clear     */
    uint32_t ood_samples;     /* out-of-domain samples per commitment         */
    uint32_t pow_bits;        /* grinding per round (0: none)                 */
    uint32_t final_pow_bits;
    uint32_t batch_size;      /* polynomials committed together: 1, 2 or 4  */
    uint32_t queries[PKO_WHIR_MAX_ROUNDS + 1]; /* STIR queries of rounds 0..R-1, final at R */
} pko_whir_params;
/* The schedule: R + 1 = max(1, ceil((n - 6) / k)) folds of k variables,
 * queries[r] = ceil((security - pow) / (rate_r / 2)) with rate_r =
 * log_inv_rate + r (k - 1) the log inverse rate of codeword r. */
int pko_whir_params_init(pko_whir_params *p, unsigned n, unsigned k, unsigned log_inv_rate,
                         unsigned security_bits, unsigned pow_bits);
size_t pko_whir_commit_words(const pko_whir_params *p);
size_t pko_whir_proof_words(const pko_whir_params *p, size_t ncov);
/* n bytes: 31 low bytes of the canonical form of each squeezed element. */
void pko_transcript_squeeze_bytes(pko_transcript *t, uint8_t *out, size_t n);
/* In place over 2^n entries: zeta: v[b | 2^i] += v[b]; mobius_t: v[b] -= v[b | 2^i]. */
void pko_subset_zeta(uint64_t *v, unsigned n);
void pko_subset_mobius_t(uint64_t *v, unsigned n);
/* Batches (the ZK commitment, RunZKWhir + parseBatchedCommitment,
 * recursive-verifier/app/circuit/whir.go:53-218, mtUtilities.go:51-119):
 * batch_size polynomials f_0..f_{B-1} of 2^n coefficients each are committed
 * in one tree whose row i holds f_0's 2^k values, then f_1's, ...: the
 * commitment of their concatenation with folding factor k + log2 B.  After
 * the OOD answers of every polynomial a batching challenge b is drawn; the
 * proof is about c = sum_i b^i f_i, with every statement's value sent per
 * polynomial, and the first codeword's openings are the wide rows, which
 * the verifier collapses with powers of b (rlcBatchedLeaves) before folding.
 *
 * The commitment: codeword (2^(n + log_inv_rate) Fr) of 2^k contiguous
 * messages and its tree over canonical leaves (2 L - 1 digests). */
int pko_whir_commit(const uint64_t *coeffs, size_t num_coeffs, unsigned k, unsigned log_inv_rate,
                    uint64_t *codeword, uint8_t *layers);
/* Absorb the root, draw the commitment's OOD points, absorb f_i(z_j)
 * (polynomial-major), and with batch_size > 1 draw the batching challenge.
 * coeffs: batch_size x 2^n (concatenated).  words: root (4) + answers
 * (4 batch_size ood); ood_points: 4 ood, then the batching challenge when
 * batch_size > 1. */
int pko_whir_commit_ood(const pko_whir_params *p, pko_transcript *t, const uint64_t *coeffs,
                        const uint8_t root[32], uint64_t *commit_words, uint64_t *ood_points);
/* The proof (pko_whir_proof_words words) of the ncov covectors (ncov x 2^n,
 * coefficient space) against the commitment (coeffs: batch_size x 2^n;
 * codeword and layers: the commitment of their concatenation). */
int pko_whir_prove(const pko_whir_params *p, pko_transcript *t, const uint64_t *coeffs,
                   const uint64_t *codeword, const uint8_t *layers, const uint64_t *commit_words,
                   const uint64_t *ood_points, const uint64_t *covectors, size_t ncov,
                   uint64_t *proof);
/* 0 when the proof is accepted, else a PKO_WHIR_REJECT_* code. */
#define PKO_WHIR_BAD_PARAMS -1
#define PKO_WHIR_REJECT_FORMAT -2
#define PKO_WHIR_REJECT_SUMCHECK -3
#define PKO_WHIR_REJECT_POW -4
#define PKO_WHIR_REJECT_MERKLE -5
#define PKO_WHIR_REJECT_FINAL_POLY -6
#define PKO_WHIR_REJECT_FINAL_CLAIM -7
int pko_whir_verify(const pko_whir_params *p, pko_transcript *t, const uint64_t *covectors,
                    size_t ncov, const uint64_t *commit_words, const uint64_t *proof,
                    size_t proof_words);
/* The two halves of pko_whir_verify, for a transcript that carries other
 * messages between the commitment and the proof: the commitment's part
 * (root, OOD points into ood_points, answers), then the proof's. */
int pko_whir_verify_commit(const pko_whir_params *p, pko_transcript *t,
                           const uint64_t *commit_words, uint64_t *ood_points);
int pko_whir_verify_proof(const pko_whir_params *p, pko_transcript *t, const uint64_t *covectors,
                          size_t ncov, const uint64_t *commit_words, const uint64_t *ood_points,
                          const uint64_t *proof, size_t proof_words);

/* The three covectors A^T eq(alpha), B^T eq(alpha), C^T eq(alpha)
 * (multiply_transposed_by_eq_alpha, provekit/common/src/utils/sumcheck.rs:206-227),
 * eq truncated to num_constraints, each zero-padded to len entries: out is
 * 3 x len Fr.  Computed as the scatter sum over the rows of M. */
int pko_r1cs_covectors(const pko_r1cs *r1cs, const uint64_t *alpha, size_t m0, size_t len,
                       uint64_t *out);
/* The whole proof's WHIR statements in the reference's order
 * (prove_from_alphas, provekit/prover/src/whir_r1cs.rs:247-301): with public
 * inputs the public weight [1, x, .., x^n] on the first n + 1 entries
 * (make_public_weight, provekit/common/src/prefix_covector.rs:173-186), then
 * A^T eq(alpha), B^T eq(alpha), C^T eq(alpha), then the blinding covector
 * expand_powers::<4>(alpha) at blinding_offset (OffsetCovector, :90-112).
 * out: (4 or 5) x len Fr; returns the count. */
int pko_r1cs_statement_covectors(const pko_r1cs *r1cs, const uint64_t public_x[4],
                                 const uint64_t *alpha, size_t m0, size_t blinding_offset,
                                 size_t len, uint64_t *out);
/* PublicInputs::hash (provekit/common/src/witness/mod.rs:86-97): 0, or
 * compress(v, 0), or the left fold of compress; canonical in and out. */
void pko_public_inputs_hash(uint64_t out[4], const uint64_t *values_canonical, size_t n);
/* WhirR1CSScheme::new_for_r1cs sizing (provekit/r1cs-compiler/src/whir_r1cs.rs:48-92). */
void pko_r1cs_sizing(size_t num_constraints, size_t num_witnesses, size_t *m, size_t *m0);
/* The synthetic satisfiable R1CS of the prove workload, generated on the
 * host without the CUDA library: w[0] = 1, w[1 ..= ni] from
 * pko_sample_fr(seed); row i: A_i and B_i hold 1-3 nonzeros (counts drawn
 * for every row first) at uniform columns in [0, ni + i] with coefficients
 * from pko_sample_fr(seed + 1), C_i = e_{ni+1+i}, w[ni+1+i] = <A_i,w><B_i,w>.
 * Integer choices from splitmix64(seed).  The reference compiles its R1CS
 * from Noir programs; this workload has no counterpart there.  Capacities as
 * for pko_r1cs: row_ptr nc+1; cols/vals 3 nc for A and B, nc for C; witness
 * 1 + ni + nc Fr (Montgomery form).  Returns 0, or -1 when the witness count
 * does not fit u32 columns. */
int pko_synthetic_r1cs(uint64_t seed, size_t nc, size_t ni, uint64_t *row_ptr[3],
                       uint32_t *cols[3], uint64_t *vals[3], size_t nnz_out[3],
                       uint64_t *witness);
/* A whole proof: pko_spartan_prove with the commitment's OOD samples drawn
 * after its root and the WHIR proof of the three zero-padded covectors
 * M^T eq(alpha) against their evaluations; whir->num_variables must be the
 * sizing's m.  out->transcript is the state the WHIR prover starts from. */
int pko_prove_r1cs(const pko_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                   uint64_t domain, const pko_whir_params *whir, pko_spartan_proof *out,
                   uint64_t *whir_commit_words, uint64_t *whir_proof);

/* ---- Two commitments: R1CS with verifier challenges -------------------
 * Sizing with the witness split at w1_size (WhirR1CSScheme::new_for_r1cs,
 * provekit/r1cs-compiler/src/whir_r1cs.rs:48-92): m = max(log w1, log w2, 13),
 * one more when w1's padding cannot hold the 4 m0 blinding coefficients.
 * w1_size = num_witnesses is pko_r1cs_sizing. */
void pko_r1cs_sizing_split(size_t num_constraints, size_t num_witnesses, size_t w1_size,
                           size_t *m, size_t *m0);

/* Fills witness[w1_size .. num_witnesses) from the challenges (Montgomery
 * form): the caller's witness solver for w2 (provekit/prover/src/lib.rs:189-212). */
typedef void (*pko_w2_solver)(void *ctx, const uint64_t *challenges, size_t num_challenges,
                              uint64_t *witness);

typedef struct {
    pko_spartan_proof spartan;  /* root, evals: w1's; transcript: where w1's WHIR proof starts */
    uint8_t root2[32];          /* w2's commitment root (canonical bytes)      */
    uint64_t evals2[3][4];      /* <M^T eq(alpha) restricted to w2, w2>, M = A, B, C */
    uint64_t challenge_eval[4]; /* <[1, x, ..], w2 at the offsets>; 0 without challenges */
} pko_dual_proof;

/* The dual-commitment proof (Prove::prove, provekit/prover/src/lib.rs:145-232,
 * then prove_from_alphas's second branch, provekit/prover/src/whir_r1cs.rs:302-425):
 *   commit w1 = witness[0, w1_size) with the blinding polynomial at w1_size
 *   (whir-ZK batch: mask from blinding_seed ^ 0x243f6a8885a308d3), squeeze
 *   num_challenges challenges, solve(ctx, ..) writes w2, commit w2 (mask from
 *   blinding_seed ^ 0x13198a2e03707344, no blinding polynomial), zk sumcheck
 *   over the whole witness, public weights, M^T eq(alpha) split at w1_size,
 *   messages evals1, evals2, public eval (with public inputs), challenge eval
 *   (with challenges), then two WHIR proofs on one transcript: w1's of
 *   [public?, A|w1, B|w1, C|w1, blinding], w2's of [A|w2, B|w2, C|w2,
 *   challenge weight?] (the challenge weight holds x^j at offsets[j], w2-relative).
 * challenges: num_challenges Fr out.  Word counts: pko_whir_commit_words and
 * pko_whir_proof_words(whir, 4 or 5) / (whir, 3 or 4). */
int pko_prove_r1cs_dual(const pko_r1cs *r1cs, size_t w1_size, const size_t *challenge_offsets,
                        size_t num_challenges, uint64_t *witness, pko_w2_solver solve, void *ctx,
                        uint64_t blinding_seed, uint64_t domain, const pko_whir_params *whir,
                        pko_dual_proof *out, uint64_t *challenges, uint64_t *commit_words1,
                        uint64_t *commit_words2, uint64_t *proof1, uint64_t *proof2);

/* A synthetic R1CS with challenges: pko_synthetic_r1cs(seed, nc1, ni) as w1
 * (w1_size = 1 + ni + nc1), then w2 of num_challenges + rows2 entries with
 * challenge j at w2 offset j * floor(w2_size / num_challenges) and the
 * products at the other offsets in order; row nc1 + i: A = the challenge
 * i mod num_challenges (the constant w[0] without challenges), B = 1-2 w1
 * columns with coefficients from pko_sample_fr(seed + 2), C = product i.
 * Capacities: row_ptr nc1 + rows2 + 1; cols/vals 3 (nc1 + rows2) for A and
 * B, nc1 + rows2 for C; witness 1 + ni + nc1 + num_challenges + rows2 Fr
 * (w2 zeroed); offsets num_challenges.  Returns 0 or -1 (too large). */
int pko_synthetic_r1cs_dual(uint64_t seed, size_t nc1, size_t ni, size_t num_challenges,
                            size_t rows2, uint64_t *row_ptr[3], uint32_t *cols[3],
                            uint64_t *vals[3], size_t nnz_out[3], uint64_t *witness,
                            size_t *challenge_offsets);
/* The solver of that instance (a pko_w2_solver): the challenges at their
 * offsets, then for rows first_row.. in order w[C col] = (A w)(B w). */
typedef struct {
    const pko_r1cs *r1cs;
    size_t w1_size, first_row;
    const size_t *challenge_offsets;
} pko_synthetic_dual;
void pko_synthetic_dual_solve(void *ctx, const uint64_t *challenges, size_t num_challenges,
                              uint64_t *witness);

int pko_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
