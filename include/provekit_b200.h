/*
 * provekit_b200.h -- C ABI of the B200 (sm_100a) ProveKit prover hot path.
 *
 * Field elements are BN254 Fr as 4 x uint64_t little-endian limbs, exactly the
 * in-memory layout of arkworks' `ark_bn254::Fr` (Montgomery form, R = 2^256,
 * fully reduced), so a Rust caller passes `slice.as_ptr() as *const u64`.
 * Skyscraper inputs/outputs are raw bytes, as in the reference's
 * `HashEngine::hash_many(&[u8], &mut [Hash])`.
 *
 * Pointer classes:
 *   pkg_*       device pointers, work enqueued on `stream` (NULL = legacy
 *               default stream); the call returns once the work is enqueued
 *               unless the entry point says otherwise.
 *   pkg_host_*  host pointers, synchronous: copy in, compute on the current
 *               device, copy out.  These are the drop-ins for the reference's
 *               host-slice plugin traits.
 *
 * Every entry point returns 0 (PKG_OK) or a negative PKG_ERR_* code and never
 * throws; pkg_last_error() returns the calling thread's last message
 * (convention of tooling/provekit-ffi/src/ffi.rs:29-95).  Where the reference
 * panics on a contract violation, the entry point returns
 * PKG_ERR_INVALID_ARGUMENT.
 */
#ifndef PROVEKIT_B200_H
#define PROVEKIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PKG_OK 0
#define PKG_ERR_INVALID_ARGUMENT (-1)
#define PKG_ERR_CUDA (-2)
#define PKG_ERR_OUT_OF_MEMORY (-3)
#define PKG_ERR_UNSUPPORTED (-4)
#define PKG_ERR_TIMEOUT (-5)

/* Leaf encodings for Merkle commits over Fr codewords. */
#define PKG_LEAF_CANONICAL 0   /* leaf bytes = canonical LE limbs (x), the   */
                               /* values the recursive verifier re-hashes   */
#define PKG_LEAF_MONTGOMERY 1  /* leaf bytes = raw in-memory limbs (x*2^256) */

typedef void *pkg_stream_t; /* a cudaStream_t */

/* ---- library ------------------------------------------------------------ */
/* Thread-local message of the last failing call on this thread ("" if none).
 * Replaces pk_get_last_error (tooling/provekit-ffi/src/ffi.rs:73-89). */
const char *pkg_last_error(void);
/* ABI version (major*10000 + minor*100 + patch). */
int pkg_version(void);

/* Seeded ChaCha20 Fr sampler for synthetic inputs: RFC 8439 block function
 * with a 64-bit block counter in words 12-13 and zero nonce, key = seed (LE)
 * in the first 8 bytes; each 64-byte block yields two 32-byte candidates,
 * masked to 254 bits and rejected if >= p.  Host memory; Montgomery form when
 * mont != 0.  No reference counterpart (the reference samples with
 * ark_std::rand::thread_rng). */
int pkg_sample_fr(uint64_t seed, size_t n, uint64_t *out, int mont);

/* ---- ntt crate (ntt/src/ntt.rs) ------------------------------------------ */
/* In-place NTT, normal order in, bit-reversed order out, over
 * len / codeword_size interleaved columns; the first log2(num_groups) stages
 * are skipped (the caller replicated cosets).
 * Replaces `pub fn ntt_nr(values: &mut [Fr], codeword_size, num_groups)`
 * (ntt/src/ntt.rs:105-108, 150-248).  Device pointer. */
int pkg_ntt_nr(uint64_t *values, size_t len, size_t codeword_size, size_t num_groups,
               pkg_stream_t stream);
/* Inverse NTT, bit-reversed order in, normal order out.
 * Replaces `pub fn intt_rn(input: &mut [Fr])` (ntt/src/ntt.rs:326-348). */
int pkg_intt_rn(uint64_t *values, size_t len, pkg_stream_t stream);
/* Grow the device-resident twiddle table to `order` (power of two <= 2^28).
 * Replaces `NTTEngine::with_order` (ntt/src/ntt.rs:39-45).  Growing builds
 * the new table synchronously (cudaMalloc + a private stream); superseded
 * tables stay allocated, so concurrent callers on other streams are safe.
 * Reserve before capturing a CUDA graph. */
int pkg_ntt_engine_reserve(size_t order);
/* pkg_intt_rn for callers that cannot let this library allocate device
 * memory (a service that reserves all HBM for its own admission control, or
 * an application whose framework allocator owns the free memory; cudaMalloc
 * and cudaFree may also synchronise the device).  No counterpart in the
 * reference.  Same result as pkg_intt_rn; calls no cudaMalloc/cudaFree or
 * allocating library routine.  Its scratch (twiddles + gather buffer) is one
 * fixed 3 MiB __device__ array in the library, held by every GPU that loads
 * it until exit, so len is limited to 2^16 (larger lengths return
 * PKG_ERR_INVALID_ARGUMENT).  All calls share that array: calls whose work
 * overlaps on the GPU (other streams, other host threads) race; serialise
 * them.  Each call writes every scratch word it reads, so no state carries
 * over between calls.  The first call on a device resolves the array's
 * device address (cudaGetSymbolAddress) with that device current; make that
 * first call before any stream capture.  Device pointer. */
int pkg_intt_rn_noalloc(uint64_t *values, size_t len, pkg_stream_t stream);
/* Host-slice forms of the two calls above (synchronous). */
int pkg_host_ntt_nr(uint64_t *values, size_t len, size_t codeword_size, size_t num_groups);
int pkg_host_intt_rn(uint64_t *values, size_t len);

/* ---- RSFr: whir ReedSolomon<Fr> plugin (provekit/common/src/ntt.rs) ----- */
/* next_order (ntt.rs:13-20): smallest power of two >= size, if <= 2^28. */
int pkg_rs_next_order(size_t size, size_t *order_out);
/* generator (ntt.rs:102-104): Fr::get_root_of_unity(codeword_length), mont. */
int pkg_rs_generator(size_t codeword_length, uint64_t out[4]);
/* evaluation_points (ntt.rs:22-42): out[i] = generator^bitrev(indices[i]).
 * Host memory. */
int pkg_rs_evaluation_points(size_t codeword_length, const size_t *indices, size_t n,
                             uint64_t *out);
/* interleaved_encode (ntt.rs:51-100).  messages: num_messages x
 * message_length Fr, message-major (message j at j*message_length); masks:
 * mask_len Fr in the reference's interleaved layout; out: codeword_length x
 * num_messages Fr (row i = the num_messages evaluations at point i).
 * Device pointers. */
int pkg_rs_interleaved_encode(const uint64_t *messages, size_t num_messages,
                              size_t message_length, const uint64_t *masks, size_t mask_len,
                              size_t codeword_length, uint64_t *out, pkg_stream_t stream);
/* Host form with the trait's `&[&[Fr]]` message list (synchronous). */
int pkg_host_rs_interleaved_encode(const uint64_t *const *messages, size_t num_messages,
                                   size_t message_length, const uint64_t *masks,
                                   size_t mask_len, size_t codeword_length, uint64_t *out);

/* ---- Skyscraper (skyscraper/core, provekit/common/src/skyscraper) ------- */
/* count two-to-one compressions of 64-byte messages into 32-byte hashes.
 * Replaces skyscraper::simple::compress_many (skyscraper/core/src/simple.rs:3-9). */
int pkg_skyscraper_compress_many(const uint8_t *messages, size_t count, uint8_t *hashes,
                                 pkg_stream_t stream);
/* SkyscraperHashEngine::hash_many (provekit/common/src/skyscraper/whir.rs:42-100):
 * size 32 copies, 64 compresses, larger multiples of 32 left-fold the chunks. */
int pkg_skyscraper_hash_many(size_t size, const uint8_t *input, size_t count,
                             uint8_t *output, pkg_stream_t stream);
int pkg_host_skyscraper_hash_many(size_t size, const uint8_t *input, size_t count,
                                  uint8_t *output);
/* Skyscraper PoW (skyscraper/core/src/generic.rs:42-71): smallest nonce with
 * compress(challenge, [nonce,0,0,0]) < threshold, searched on the device with
 * every candidate below the answer evaluated.  Host in/out, synchronous. */
int pkg_skyscraper_pow_solve(const uint64_t challenge[4], const uint64_t threshold[4],
                             uint64_t *nonce_out);

/* ---- Poseidon2 (poseidon2/src), BN254, t = 4, rf = 8, rp = 56 ------------ */
/* In-place permutation of n states of 4 Fr (Montgomery form), state i at
 * states[16*i .. 16*i + 16).  Replaces poseidon2_permutation
 * (poseidon2/src/permutation.rs:134-177).  Device pointer. */
int pkg_poseidon2_permutation_many(uint64_t *states, size_t n, pkg_stream_t stream);
/* out[i] = poseidon2_hash(inputs[i*len .. (i+1)*len)) (poseidon2/src/hash.rs:17-47:
 * rate 3, capacity lane initialised to len * 2^64).  Device pointers. */
int pkg_poseidon2_hash_many(const uint64_t *inputs, size_t len, size_t n, uint64_t *out,
                            pkg_stream_t stream);

/* ---- Merkle commit ------------------------------------------------------- */
/* Binary Skyscraper Merkle tree over num_leaves (power of two) leaves of
 * leaf_size bytes: leaf digests = hash_many(leaf_size), internal nodes =
 * hash_many(64) of (left || right).  layers receives 2*num_leaves-1 digests
 * level by level: leaf digests first, root last.  Device pointers. */
int pkg_merkle_tree(const uint8_t *leaves, size_t leaf_size, size_t num_leaves,
                    uint8_t *layers, pkg_stream_t stream);
/* Same tree with leaf i = the fr_per_leaf Fr of codeword row i (the
 * interleaved_encode output), encoded per PKG_LEAF_*.  Device pointers. */
int pkg_merkle_tree_fr(const uint64_t *codeword, size_t fr_per_leaf, size_t num_leaves,
                       int leaf_encoding, uint8_t *layers, pkg_stream_t stream);

/* The two halves of pkg_merkle_tree_fr: leaf digests into layers[0..L), then
 * the internal levels above them (layers must hold 2*L-1 digests). */
int pkg_merkle_leaves_fr(const uint64_t *codeword, size_t fr_per_leaf, size_t num_leaves,
                         int leaf_encoding, uint8_t *layers, pkg_stream_t stream);
int pkg_merkle_levels(uint8_t *layers, size_t num_leaves, pkg_stream_t stream);

/* WHIR commit of one multilinear polynomial: the coefficients are split into
 * 2^folding_factor contiguous messages, Reed-Solomon encoded at rate
 * 2^-log_inv_rate (interleaved_encode), and committed with
 * pkg_merkle_tree_fr.  codeword_out: num_coeffs << log_inv_rate Fr;
 * layers_out: 2*L-1 digests, L = (num_coeffs >> folding_factor) << log_inv_rate.
 * Device pointers. */
int pkg_whir_commit(const uint64_t *coeffs, size_t num_coeffs, unsigned folding_factor,
                    unsigned log_inv_rate, const uint64_t *masks, size_t mask_len,
                    int leaf_encoding, uint64_t *codeword_out, uint8_t *layers_out,
                    pkg_stream_t stream);

/* ---- Spartan sumcheck side (provekit/common/src/utils/sumcheck.rs,
 *      provekit/prover/src/whir_r1cs.rs) -------------------------------- */
/* Fiat-Shamir transcript.  The reference's is spongefish's DuplexSponge over
 * skyscraper::reference::permute (provekit/common/src/skyscraper/sponge.rs:27-41,
 * transcript_sponge.rs:19-111); spongefish is not available, so this is a
 * minimal duplex over the same permutation: state (l, r) canonical;
 * init: l = domain mod p, r = 0, permute; absorb(x): l += x (canonical),
 * permute; squeeze: permute, return l (Montgomery form).  Host only. */
typedef struct {
  uint64_t l[4];
  uint64_t r[4];
} pkg_transcript;
int pkg_transcript_init(pkg_transcript *t, const uint64_t domain[4]);
int pkg_transcript_absorb(pkg_transcript *t, const uint64_t x[4]);
int pkg_transcript_squeeze(pkg_transcript *t, uint64_t out[4]);

/* eq(r, x) for x < num_entries over the nr-variable hypercube, r_0 on the
 * most significant bit (calculate_evaluations_over_boolean_hypercube_for_eq,
 * sumcheck.rs:108-153).  r: host; out: device. */
int pkg_eq_hypercube(const uint64_t *r, size_t nr, size_t num_entries, uint64_t *out,
                     pkg_stream_t stream);
/* One round of the Spartan map-reduce (the closure at whir_r1cs.rs:551-559 over
 * sumcheck_fold_map_reduce, sumcheck.rs:14-102) on device tables a, b, c, eq of
 * length size.  fold (host, or NULL): fold the top variable first in the
 * quarter layout (tables then hold size/2 live entries).  out (host): f(0),
 * f(-1), f(inf).  Synchronous. */
int pkg_spartan_round(uint64_t *a, uint64_t *b, uint64_t *c, uint64_t *eq, size_t size,
                      const uint64_t *fold, uint64_t out[12], pkg_stream_t stream);
/* run_zk_sumcheck_prover (whir_r1cs.rs:519-621): m0 rounds over device tables
 * a, b, c of length 2^m0 (modified in place), blinding polynomial g (host,
 * m0 x 4 Fr), w1_blinding = w1[offset .. offset + 4*m0] (host).  Drives the
 * transcript (in/out) and returns r (m0), rho, sum_g, the 4*m0 round
 * coefficients, alpha (m0) and the blinding evaluation (all host).
 * Synchronous (one device->host read of 3 Fr per round). */
int pkg_spartan_sumcheck(uint64_t *a, uint64_t *b, uint64_t *c, size_t m0, const uint64_t *g,
                         const uint64_t *w1_blinding, pkg_transcript *transcript,
                         uint64_t *r_out, uint64_t rho_out[4], uint64_t sum_g_out[4],
                         uint64_t *coeffs_out, uint64_t *alpha_out, uint64_t blinding_eval[4],
                         pkg_stream_t stream);
/* y = M x for a CSR matrix with one Fr per nonzero (HydratedSparseMatrix *
 * &[Fr], provekit/common/src/sparse_matrix.rs:606-627); x has num_cols
 * entries.  A column index >= num_cols (a reference panic) is skipped on the
 * device and reported as PKG_ERR_INVALID_ARGUMENT.  Device pointers;
 * synchronous (reads back that flag). */
int pkg_spmv_csr(const uint64_t *row_ptr, const uint32_t *cols, const uint64_t *vals,
                 size_t num_rows, size_t num_cols, const uint64_t *x, uint64_t *y,
                 pkg_stream_t stream);
/* CSR transpose (SparseMatrix::transpose, sparse_matrix.rs:409): row_ptr_t
 * has num_cols + 1 entries; the order of entries inside a transposed row is
 * unspecified (SpMV results do not depend on it).  Out-of-range column
 * indices are skipped and reported as PKG_ERR_INVALID_ARGUMENT.  Device
 * pointers; synchronous. */
int pkg_csr_transpose(const uint64_t *row_ptr, const uint32_t *cols, const uint64_t *vals,
                      size_t num_rows, size_t num_cols, size_t nnz, uint64_t *row_ptr_t,
                      uint32_t *cols_t, uint64_t *vals_t, pkg_stream_t stream);
/* c[i] = a[i] * b[i] for i < n, 0 for n <= i < padded (calculate_witness_bounds,
 * sumcheck.rs:163-179).  Device pointers. */
int pkg_hadamard_pad(const uint64_t *a, const uint64_t *b, size_t n, size_t padded,
                     uint64_t *c, pkg_stream_t stream);
/* sum_i a[i] * b[i] (whir::algebra::dot as used at whir_r1cs.rs:614-617, 637,
 * 650).  a, b device; out host; synchronous. */
int pkg_dot(const uint64_t *a, const uint64_t *b, size_t n, uint64_t out[4], pkg_stream_t stream);

/* ---- Spartan prove core ---------------------------------------------------- */
/* An R1CS instance as three CSR matrices (num_constraints x num_witnesses, one
 * Fr per nonzero, hydrated).  Device pointers. */
typedef struct {
  size_t num_constraints, num_witnesses;
  const uint64_t *row_ptr[3]; /* A, B, C; num_constraints + 1 entries each */
  const uint32_t *cols[3];
  const uint64_t *vals[3];
  size_t nnz[3];
  size_t num_public_inputs;   /* the public inputs are witness[1 ..= this] */
  /* Optional, all three or none: the transposes of A, B, C (num_witnesses
   * rows: row_ptr_t num_witnesses + 1 entries, cols_t / vals_t nnz[k]
   * entries, column indices < num_constraints), built once for a resident
   * circuit with
   * pkg_r1cs_build_transposes or pkg_csr_transpose
   * (transpose_r1cs_matrices, provekit/common/src/utils/sumcheck.rs:195-206).
   * NULL: every proof transposes the matrices itself. */
  const uint64_t *row_ptr_t[3];
  const uint32_t *cols_t[3];
  const uint64_t *vals_t[3];
} pkg_r1cs;

/* Bytes of device memory the three transposes of r1cs take (row pointers,
 * columns and values, each 256-byte aligned).  Host only. */
size_t pkg_r1cs_transposes_bytes(const pkg_r1cs *r1cs);
/* Builds the three transposes into buf (device, pkg_r1cs_transposes_bytes
 * long, 256-byte aligned) and points r1cs->row_ptr_t / cols_t / vals_t into
 * it.  Synchronous.  Out-of-range column indices are reported as
 * PKG_ERR_INVALID_ARGUMENT. */
int pkg_r1cs_build_transposes(pkg_r1cs *r1cs, void *buf, pkg_stream_t stream);

/* Everything the prover produces before WHIR's own prove rounds. */
typedef struct {
  size_t m, m0;                  /* committed variables, sumcheck variables */
  uint8_t root[32];              /* Merkle root of the witness commitment  */
  uint64_t r[30][4];             /* eq challenges (m0)                     */
  uint64_t coeffs[120][4];       /* 4 round coefficients per round (4*m0) */
  uint64_t alpha[30][4];         /* sumcheck challenges (m0)               */
  uint64_t rho[4], sum_g[4], blinding_eval[4], public_x[4];
  uint64_t evals[3][4];          /* <A^T eq(alpha), w>, <B^T ...>, <C^T ...> */
  pkg_transcript transcript;     /* state after the last message           */
  uint64_t public_hash[4];       /* PublicInputs::hash (canonical; 0 if none) */
  uint64_t public_eval[4];       /* <[1, x, .., x^n], w> (0 if no publics)   */
} pkg_spartan_proof;

/* The prover's work up to WHIR's prove call for a single-commitment R1CS
 * (no public inputs, no challenges): WhirR1CSScheme::new_for_r1cs sizing
 * (provekit/r1cs-compiler/src/whir_r1cs.rs:48-92); WhirR1CSProver::commit
 * (provekit/prover/src/whir_r1cs.rs:82-140) with the 4*m0 blinding
 * coefficients drawn from pkg_sample_fr(blinding_seed) instead of thread_rng
 * and the commitment = pkg_whir_commit(folding_factor, log_inv_rate,
 * canonical leaves) of the padded witness, root absorbed; prove_noir
 * (:143-187): witness bounds, zk sumcheck, eq(alpha), transposed SpMV;
 * prove_from_alphas (:247-301): public-weight challenge (hash of no public
 * inputs = 0), the three covector evaluations absorbed.  witness: device,
 * num_witnesses Fr.  Synchronous. */
int pkg_spartan_prove(const pkg_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                      uint64_t transcript_domain, unsigned folding_factor, unsigned log_inv_rate,
                      pkg_spartan_proof *out, pkg_stream_t stream);

/* Per-stage host wall-clock (ms) of the calling thread's last
 * pkg_spartan_prove or pkg_prove_r1cs: [0] commit (to the root, and the
 * OOD answers), [1] witness bounds, [2] zk sumcheck, [3] eq(alpha) + public
 * weight, [4] transposed products and evaluations, [5] the WHIR proof (0
 * for pkg_spartan_prove).  The witness bounds are only enqueued (their
 * device time falls in [2]); every other stage ends with a synchronisation.
 * No counterpart in the reference (diagnostics). */
#define PKG_PROVE_STAGES 6
int pkg_last_prove_stages(double ms[PKG_PROVE_STAGES]);

/* WhirR1CSScheme::new_for_r1cs sizing (provekit/r1cs-compiler/src/whir_r1cs.rs:48-92):
 * m = max(ceil log2 num_witnesses, 13), plus one when fewer than 4 m0 slots
 * are free for the blinding coefficients; m0 = max(ceil log2
 * num_constraints, 1).  Host only. */
int pkg_r1cs_sizing(size_t num_constraints, size_t num_witnesses, size_t *m, size_t *m0);

/* Synthetic satisfiable R1CS (host memory), the workload of the 2^20-constraint
 * prove benchmark: w[0] = 1, w[1..num_inputs] from pkg_sample_fr(seed); row
 * i: A_i and B_i each hold 1-3 nonzeros at uniform columns in
 * [0, num_inputs + i] with uniform Fr coefficients, C_i = e_{num_inputs+1+i},
 * and w[num_inputs+1+i] = <A_i, w> * <B_i, w>.  Integer choices come from
 * splitmix64(seed), coefficients from pkg_sample_fr(seed + 1).  Capacities:
 * row_ptr[k] num_constraints+1, cols/vals of A and B 3*num_constraints, of C
 * num_constraints; witness 1 + num_inputs + num_constraints Fr.  No
 * reference counterpart (the reference compiles R1CS from Noir programs). */
int pkg_synthetic_r1cs(uint64_t seed, size_t num_constraints, size_t num_inputs,
                       uint64_t *row_ptr[3], uint32_t *cols[3], uint64_t *vals[3],
                       size_t nnz_out[3], uint64_t *witness);
/* Synthetic R1CS with verifier challenges (host memory), the workload of
 * the two-commitment prove: pkg_synthetic_r1cs(seed, nc1, num_inputs) as
 * w1 (w1_size = 1 + num_inputs + nc1), then w2 of num_challenges + rows2
 * entries: challenge j at w2 offset j * floor(w2_size / num_challenges)
 * (offsets out), products at the other offsets in order.  Row nc1 + i: A =
 * the challenge i mod num_challenges (w[0] without challenges), B = 1-2
 * uniform w1 columns (splitmix64(seed ^ 0xd1b54a32d192ed03)) with
 * coefficients from pkg_sample_fr(seed + 2), C = product i.  Capacities:
 * row_ptr nc1 + rows2 + 1; cols/vals 3 (nc1 + rows2) for A and B,
 * nc1 + rows2 for C; witness w1_size + num_challenges + rows2 Fr (w2
 * zeroed).  No reference counterpart (the reference compiles such circuits
 * from Noir programs). */
int pkg_synthetic_r1cs_dual(uint64_t seed, size_t nc1, size_t num_inputs, size_t num_challenges,
                            size_t rows2, uint64_t *row_ptr[3], uint32_t *cols[3],
                            uint64_t *vals[3], size_t nnz_out[3], uint64_t *witness,
                            size_t *offsets);
/* That instance's w2 from the challenges (host, in place in witness): the
 * challenges at w1_size + offsets[j], then for rows first_row.. in order
 * w[C's column] = <A_row, w> <B_row, w>. */
int pkg_synthetic_dual_solve(size_t num_constraints, size_t first_row,
                             const uint64_t *const row_ptr[3], const uint32_t *const cols[3],
                             const uint64_t *const vals[3], size_t w1_size, const size_t *offsets,
                             size_t num_challenges, const uint64_t *challenges, uint64_t *witness);

/* ---- Batched form ----------------------------------------------------------- */
/* A batch of independent jobs of uneven sizes.  Job j (size n = 2^log_n,
 * 4 <= log_n <= 24) has n coefficients from pkg_sample_fr(seed + j) and runs
 *   (1) ntt_nr over a copy of its coefficients (pkg_ntt_nr),
 *   (2) the WHIR commit of its coefficients: 8 contiguous messages, rate 1/4,
 *       canonical leaves of 8 Fr (pkg_whir_commit with folding factor 3),
 *   (3) the Spartan zk-sumcheck (pkg_spartan_sumcheck) over a = its
 *       coefficients, b = its NTT output, c = the first n codeword entries,
 *       with blinding g = pkg_sample_fr(seed + 0x100000 + j), w1 blinding
 *       values = pkg_sample_fr(seed + 0x200000 + j), transcript domain j + 1.
 * Each phase runs as one grouped kernel over all jobs and the transcript runs
 * on the device, so the batch is one CUDA graph; results equal the plain
 * entry points run job by job.  No reference counterpart (the reference
 * proves one instance at a time). */
typedef struct pkg_batch pkg_batch;
typedef struct {
  uint32_t log_n;
  size_t n;
  uint64_t *coeffs, *ntt, *codeword; /* device: n, n, 4n Fr */
  uint8_t *layers;                   /* device: 2*num_leaves - 1 digests */
  size_t num_leaves;
  uint64_t transcript_domain;
  uint64_t g[120][4];            /* host copy: blinding polynomial, 4*m0 Fr  */
  uint64_t w1_blinding[120][4];  /* host copy: w1 blinding values, 4*m0 Fr  */
} pkg_batch_job;
typedef struct {
  size_t m0;
  uint64_t r[30][4], coeffs[120][4], alpha[30][4];
  uint64_t rho[4], sum_g[4], blinding_eval[4];
  pkg_transcript transcript;
} pkg_sumcheck_result;
int pkg_batch_create(const uint32_t *log_sizes, size_t njobs, uint64_t seed, pkg_batch **out);
void pkg_batch_destroy(pkg_batch *batch);
int pkg_batch_job_info(pkg_batch *batch, size_t job, pkg_batch_job *out);
/* NTT plan: passes of at most kmax stages (radix 2^kmax), 2^log_elems_per_cta
 * elements staged per CTA.  Re-planning drops a captured graph. */
int pkg_batch_set_params(pkg_batch *batch, int kmax, int log_elems_per_cta);
/* Butterflies each thread of an NTT pass runs per stage: 2^log_bpt (0..2), so
 * a CTA staging E elements has E / 2^(1 + log_bpt) threads (at least 32, at
 * most 512).  No counterpart in the reference (its NTT is a CPU crate). */
int pkg_batch_set_butterflies_per_thread(pkg_batch *batch, int log_bpt);
/* The plan's current (kmax, log2 elements per CTA, log2 butterflies per
 * thread), e.g. after pkg_batch_tune.  No counterpart in the reference. */
int pkg_batch_get_params(pkg_batch *batch, int *kmax, int *log_elems_per_cta,
                         int *log_butterflies_per_thread);
/* Autotuner: times every (kmax in 4..11, elements per CTA, butterflies per
 * thread) on this batch and keeps the fastest. */
int pkg_batch_tune(pkg_batch *batch, pkg_stream_t stream, int *best_kmax, int *best_log_elems,
                   double *best_ms);
/* Run the batch on stream.  use_graph: the first call captures the batch as
 * a CUDA graph (stream must not be the legacy default stream), later calls
 * replay it. */
int pkg_batch_run(pkg_batch *batch, int use_graph, pkg_stream_t stream);
/* Host copy of job j's sumcheck outputs (synchronous). */
int pkg_batch_sumcheck_result(pkg_batch *batch, size_t job, pkg_sumcheck_result *out);

/* ---- Served form -------------------------------------------------------------- */
/* A proving service on the current device: requests (host R1CS + witness) are
 * queued, admitted by their estimated HBM footprint within hbm_budget_bytes
 * and max_inflight slots, and proved with pkg_spartan_prove (or, with WHIR
 * parameters, pkg_prove_r1cs) by one worker
 * thread + CUDA stream per slot, so admitted jobs overlap on the device and
 * their R1CS, witness, codeword, tree and tables stay resident until done.
 * Latencies are measured from submit to completion.  No reference
 * counterpart (the reference proves one request per call,
 * tooling/provekit-ffi/src/ffi.rs:536-595). */
typedef struct pkg_server pkg_server;
typedef struct {
  size_t num_constraints, num_witnesses;
  const uint64_t *row_ptr[3]; /* host CSR A, B, C */
  const uint32_t *cols[3];
  const uint64_t *vals[3];
  size_t nnz[3];
  const uint64_t *witness;    /* host, num_witnesses Fr */
  uint64_t blinding_seed, transcript_domain;
  unsigned folding_factor, log_inv_rate;
  /* Optional whole proof (pkg_prove_r1cs): WHIR parameters for the R1CS's
   * m (their folding factor and rate replace the two above) and host
   * buffers of pkg_whir_commit_words / pkg_whir_proof_words(whir, 3) words,
   * written before pkg_server_wait returns.  NULL: the Spartan part only
   * (pkg_spartan_prove). */
  const struct pkg_whir_params_s *whir;
  uint64_t *whir_commit_words, *whir_proof;
  size_t num_public_inputs;   /* witness[1 ..= this] are public */
} pkg_prove_request;
typedef struct {
  uint64_t submit_ns, admit_ns, done_ns; /* steady clock */
  size_t footprint_bytes;                /* admission estimate */
} pkg_request_times;
typedef struct {
  size_t completed, queued, inflight;
  size_t reserved_bytes, peak_reserved_bytes;
  double p50_ms, p99_ms, p999_ms, proofs_per_s;
} pkg_server_stats;
int pkg_server_create(size_t hbm_budget_bytes, int max_inflight, pkg_server **out);
/* Queues the request without copying it: the caller's host buffers must stay
 * valid and unchanged until pkg_server_wait returns for the returned id (the
 * worker uploads them when the request is admitted).  A request whose
 * estimate exceeds the whole budget returns PKG_ERR_OUT_OF_MEMORY; row
 * pointers that do not start at 0, decrease or do not end at nnz return
 * PKG_ERR_INVALID_ARGUMENT (column indices are checked on the device: an
 * out-of-range one fails the request). */
int pkg_server_submit(pkg_server *server, const pkg_prove_request *req, uint64_t *request_id);
/* Blocks until the request is done; returns its status. */
int pkg_server_wait(pkg_server *server, uint64_t request_id, pkg_spartan_proof *proof,
                    pkg_request_times *times);
int pkg_server_get_stats(pkg_server *server, pkg_server_stats *out);
/* Finishes admitted work, fails queued requests, joins the workers. */
void pkg_server_destroy(pkg_server *server);

/* ---- WHIR prove rounds: the data-parallel operations ---------------------
 * The WHIR prover is inside the un-vendored `whir` crate (called at
 * provekit/prover/src/whir_r1cs.rs:295-301, 378-414); these are the device
 * operations its rounds are made of.  Their arithmetic follows the
 * reference's WHIR verifier restated in Go (recursive-verifier/app/...), cited
 * per function.  Fr values are Montgomery form; "host" arrays are read or
 * written synchronously, device arrays are 16-byte aligned. */
/* out[i] = sum_j w_j coeffs[j (n >> k) + i], w_j = prod_t alpha[t]^(bit t of j)
 * (MultivarPoly's weights, recursive-verifier/app/utilities/utilities.go:16-23):
 * the polynomial whose RS codeword is the fold of the 2^k-message interleaved
 * codeword.  k <= 6; n a power of two >= 2^k; alpha: host, k Fr.  Async. */
int pkg_whir_fold_coeffs(const uint64_t *coeffs, size_t n, unsigned k, const uint64_t *alpha,
                         uint64_t *out, pkg_stream_t stream);
/* out[i] = MultivarPoly(rows[i 2^k .. (i+1) 2^k), alpha): computeFold
 * (recursive-verifier/app/circuit/whir_utilities.go:182-188) over nrows rows
 * of a codeword.  k <= 6; alpha: host.  Async. */
int pkg_whir_fold_rows(const uint64_t *rows, size_t nrows, unsigned k, const uint64_t *alpha,
                       uint64_t *out, pkg_stream_t stream);
/* out[j] = sum_i coeffs[i] points[j]^i (UnivarPoly, utilities.go:25-39): the
 * out-of-domain answers.  coeffs: device, n Fr; points, out: host, npts Fr.
 * Synchronous. */
int pkg_poly_eval_many(const uint64_t *coeffs, size_t n, const uint64_t *points, size_t npts,
                       uint64_t *out, pkg_stream_t stream);
/* Authentication paths in a layers array (leaves first, root last, as
 * pkg_merkle_tree writes it): paths[q][l] = node (indices[q] >> l) ^ 1 of
 * level l, l < log2(num_leaves) -- path[0] is the leaf's sibling, the rest
 * the auth path that verifyMerkleTreeProofs walks
 * (recursive-verifier/app/circuit/whir_utilities.go:14-47).  indices, paths:
 * host (nq x log2(num_leaves) x 32 bytes).  Synchronous. */
int pkg_merkle_open(const uint8_t *layers, size_t num_leaves, const uint64_t *indices, size_t nq,
                    uint8_t *paths, pkg_stream_t stream);
/* rows[q] = codeword row indices[q] (fr_per_row Fr each): the opened leaves'
 * values.  indices, rows: host.  Synchronous. */
int pkg_gather_rows(const uint64_t *codeword, size_t fr_per_row, size_t num_rows,
                    const uint64_t *indices, size_t nq, uint64_t *rows, pkg_stream_t stream);
/* getStirChallenges (whir_utilities.go:49-79) for a power-of-two folded
 * domain: per query ceil(log2(size) / 8) big-endian challenge bytes, reduced
 * to the low log2(size) bits.  Host. */
int pkg_stir_indices(const uint8_t *bytes, size_t folded_domain_size, size_t nq, uint64_t *out);
/* One round of WHIR's weighted sumcheck over device tables f, w of size
 * entries (top variable first).  fold (host, or NULL): first fold the top
 * variable, t[i] += fold (t[i + size/2] - t[i]) (quarter layout, as
 * pkg_spartan_round); then out = (h(0), h(1), h(2)) of
 * h(X) = sum_b f(X, b) w(X, b), the evaluation form that
 * EvaluateQuadraticPolynomialFromEvaluationList and CheckSumOverBool read
 * (utilities.go:149-171).  Synchronous. */
int pkg_whir_sumcheck_round(uint64_t *f, uint64_t *w, size_t size, const uint64_t *fold,
                            uint64_t out[12], pkg_stream_t stream);
/* w[b] += sum_j coeffs[j] eq(points[j], b) for b < 2^nv (coordinate 0 on the
 * top bit of b, as pkg_eq_hypercube): the weight update for new OOD and STIR
 * constraints (computeWPoly's terms, whir_utilities.go:128-161).  w: device;
 * points (npts x nv Fr), coeffs (npts Fr): host.  Synchronous. */
int pkg_eq_accumulate(uint64_t *w, size_t nv, const uint64_t *points, const uint64_t *coeffs,
                      size_t npts, pkg_stream_t stream);

/* ---- WHIR prover: the round loop -----------------------------------------
 * Replaces the un-vendored whir crate's prove (called at
 * provekit/prover/src/whir_r1cs.rs:295-301, 378-414) for linear statements
 * <a_k, c> = v_k about a committed coefficient vector c of 2^n Fr.  The
 * proof is what the reference's Go verifier walks (runWhir,
 * recursive-verifier/app/circuit/whir.go:587-724): statement values, the
 * initial sumcheck, per round a root, OOD answers, PoW nonce, STIR openings
 * of the previous codeword (rows then authentication paths) and k sumcheck
 * messages, then the final coefficients, PoW, openings and sumcheck -- a
 * flat array of u64 words (Fr as 4 Montgomery limbs, digests as 4 LE words,
 * nonces as one word), pkg_whir_proof_words long.  Conventions the crate
 * would fix and that are chosen here: query points
 * RSFr::evaluation_points (provekit/common/src/ntt.rs:22-42); 2^k contiguous
 * messages per codeword row, so a sumcheck binds the top coefficient bit
 * first; the sumcheck runs over zeta(c) (subset sums) against
 * mobius^T(sum gamma^j a_j) (superset differences); the transcript stand-in
 * above, with bytes taken 31 per squeezed element; PoW threshold
 * floor(p / 2^bits) (CheckPoW, recursive-verifier/app/utilities/utilities.go:104-139). */
#define PKG_WHIR_MAX_ROUNDS 16
typedef struct pkg_whir_params_s {
  uint32_t num_variables;   /* n: the committed vector has 2^n entries     */
  uint32_t folding_factor;  /* k, 1..6                                      */
  uint32_t log_inv_rate;    /* starting rate 2^-log_inv_rate (1..8)         */
  uint32_t num_rounds;      /* R: rounds that commit a folded polynomial    */
  uint32_t final_vars;      /* n - (R+1) k, sent as 2^final_vars coeffs     */
  uint32_t ood_samples;     /* OOD samples per commitment (0..4)            */
  uint32_t pow_bits;        /* grinding per round (0..27, 0 = none)         */
  uint32_t final_pow_bits;
  uint32_t batch_size;      /* polynomials committed together: 1, 2 or 4  */
  uint32_t queries[PKG_WHIR_MAX_ROUNDS + 1]; /* rounds 0..R-1, final at R   */
} pkg_whir_params;
/* Schedule: R + 1 = max(1, ceil((n - 6) / k)) folds; queries[r] =
 * ceil(2 (security - pow) / rate_r), rate_r = log_inv_rate + r (k - 1);
 * batch_size 1.
 * Batches (whir's ZK commitment, as the reference's Go verifier reads it:
 * RunZKWhir and parseBatchedCommitment, recursive-verifier/app/circuit/whir.go:53-218,
 * mtUtilities.go:51-119): batch_size polynomials f_i of 2^n coefficients are
 * committed in one tree whose row holds f_0's 2^k values, then f_1's, ...
 * (pkg_whir_commit of their concatenation with folding factor k +
 * log2 batch_size); after every polynomial's OOD answers a batching
 * challenge b is drawn, the statement values are sent per polynomial, the
 * rounds prove c = sum_i b^i f_i, and the first codeword's openings are the
 * wide rows. */
int pkg_whir_params_init(pkg_whir_params *p, unsigned num_variables, unsigned folding_factor,
                         unsigned log_inv_rate, unsigned security_bits, unsigned pow_bits);
size_t pkg_whir_commit_words(const pkg_whir_params *p);
/* 0 for invalid parameters. */
size_t pkg_whir_proof_words(const pkg_whir_params *p, size_t num_covectors);
/* n challenge bytes: the 31 low bytes of each squeezed element's canonical
 * little-endian form. */
int pkg_transcript_squeeze_bytes(pkg_transcript *t, uint8_t *out, size_t n);
/* In place over 2^n device entries: ZETA v[b | 2^i] += v[b] (coefficients ->
 * hypercube evaluations); MOBIUS_T v[b] -= v[b | 2^i] (its adjoint inverse:
 * a covector on coefficients -> a weight on the hypercube).  Async. */
#define PKG_SUBSET_ZETA 0
#define PKG_SUBSET_MOBIUS_T 1
int pkg_subset_transform(uint64_t *v, unsigned n, int mode, pkg_stream_t stream);
/* The commitment's transcript part, after pkg_whir_commit(coeffs,
 * batch_size 2^n, folding_factor + log2 batch_size, log_inv_rate, no masks,
 * PKG_LEAF_CANONICAL): absorb the root, draw ood_samples points, absorb
 * f_i(z_j) polynomial by polynomial, and for a batch draw the batching
 * challenge.  coeffs (batch_size x 2^n, concatenated), layers: device;
 * commit_words (4 + 4 ood_samples batch_size: root, answers), ood_points
 * (ood_samples, then the batching challenge for a batch): host.
 * Synchronous. */
int pkg_whir_commit_ood(const pkg_whir_params *p, pkg_transcript *t, const uint64_t *coeffs,
                        const uint8_t *layers, uint64_t *commit_words, uint64_t *ood_points,
                        pkg_stream_t stream);
/* The proof of num_covectors (<= 16) statements: covectors device
 * (num_covectors x 2^n Fr, coefficient space); coeffs (batch_size x 2^n),
 * codeword, layers the commitment (device); ood_points from
 * pkg_whir_commit_ood; proof: host, pkg_whir_proof_words words.
 * Synchronous; t advances past the proof. */
int pkg_whir_prove(const pkg_whir_params *p, pkg_transcript *t, const uint64_t *coeffs,
                   const uint64_t *codeword, const uint8_t *layers, const uint64_t *ood_points,
                   const uint64_t *covectors, size_t num_covectors, uint64_t *proof,
                   pkg_stream_t stream);
/* Per-phase host wall-clock (ms) of the calling thread's last WHIR prove:
 * [0] set-up (subset transforms, statement values, weight table), [1]
 * sumcheck rounds, [2] folds + commitments + roots, [3] OOD answers, [4] PoW,
 * [5] STIR openings, [6] weight updates, [7] the final polynomial.  A phase
 * that ends without a synchronisation leaves its device time to the next
 * one that synchronises.  Diagnostics; no reference counterpart. */
#define PKG_WHIR_STAGES 8
int pkg_last_whir_stages(double ms[PKG_WHIR_STAGES]);

/* A whole proof (WhirR1CSProver::prove_noir with whir's prove,
 * provekit/prover/src/whir_r1cs.rs:143-301): pkg_spartan_prove's work with
 * whir's commitment OOD samples drawn right after the root
 * (pkg_whir_commit_ood: whir_commit_words), then pkg_whir_prove of the
 * single-commitment statements in the reference's order (prove_from_alphas,
 * :258-301): the public weight [1, x, .., x^n] on the first n + 1 entries
 * when there are n public inputs (make_public_weight,
 * provekit/common/src/prefix_covector.rs:173-186), A^T eq(alpha),
 * B^T eq(alpha), C^T eq(alpha) (zero-padded to 2^m), and the blinding
 * covector expand_powers::<4>(alpha) at the blinding offset (OffsetCovector)
 * with the zk-sumcheck's blinding_eval as its value -- whir_proof:
 * pkg_whir_proof_words(whir, 4 + (n > 0)) words.  With batch_size 2
 * (whir-ZK) the witness is committed with a blinding polynomial drawn by
 * pkg_sample_fr_indexed.  whir: pkg_whir_params for pkg_r1cs_sizing's m
 * (folding factor and rate are taken from it).  out->transcript is the state
 * the WHIR prover starts from.  Synchronous. */
int pkg_prove_r1cs(const pkg_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                   uint64_t transcript_domain, const pkg_whir_params *whir,
                   pkg_spartan_proof *out, uint64_t *whir_commit_words, uint64_t *whir_proof,
                   pkg_stream_t stream);

/* ---- Two commitments: R1CS with verifier challenges ----------------------
 * The witness is split at w1_size.  w1 = witness[0, w1_size) is committed
 * first, verifier challenges are drawn from the transcript, the caller
 * solves w2 = witness[w1_size, num_witnesses) with them, w2 is committed,
 * and the proof ends with two WHIR proofs on one transcript.  This is
 * Prove::prove's flow (provekit/prover/src/lib.rs:145-232: commit w1, solve
 * w2 whose WitnessBuilder::Challenge entries squeeze the transcript,
 * prover/src/witness/witness_builder.rs:167-170, commit w2) and
 * prove_from_alphas's dual-commitment branch
 * (provekit/prover/src/whir_r1cs.rs:302-425).  It is split in two calls
 * because witness solving stays with the caller:
 *
 *   pkg_dual_prove_begin   w1's commitment (with the blinding polynomial at
 *                          w1_size; whir-ZK mask from blinding_seed as in
 *                          pkg_prove_r1cs), then num_challenges challenges
 *   (caller)               solves w2; the challenge values sit in w2 at
 *                          challenge_offsets (w2-relative, scheme.challenge_offsets)
 *   pkg_dual_prove_finish  w2's commitment (no blinding polynomial; its mask
 *                          from blinding_seed ^ 0x13198a2e03707344), the zk
 *                          sumcheck over the whole witness, public weights,
 *                          A^T eq, B^T eq, C^T eq split at w1_size, messages
 *                          evals (w1), evals2 (w2), public eval (public
 *                          inputs, on w1), challenge eval (challenges, on
 *                          w2), then WHIR proof 1 of w1's statements
 *                          [public weight?, A|w1, B|w1, C|w1, blinding] and
 *                          WHIR proof 2 of w2's [A|w2, B|w2, C|w2,
 *                          challenge weight?] (make_challenge_weight:
 *                          x^j at challenge_offsets[j], repeated offsets add)
 *   pkg_dual_prove_free    releases the state (any time; NULL is a no-op;
 *                          it synchronises the stream given to begin, which
 *                          must still exist)
 *
 * Sizing: pkg_r1cs_sizing_split.  whir: parameters for its m; batch_size 1,
 * or 2 for whir-ZK (each commitment with its own mask polynomial). */
typedef struct pkg_dual_prove pkg_dual_prove;
typedef struct {
  pkg_spartan_proof spartan; /* root, evals: w1's; transcript: where WHIR proof 1 starts */
  uint8_t root2[32];         /* w2's commitment root                       */
  uint64_t evals2[3][4];     /* <M^T eq(alpha) restricted to w2, w2>, M = A, B, C */
  uint64_t challenge_eval[4];/* <[1, x, ..], w2 at the offsets> (0 without challenges) */
} pkg_dual_proof;
/* WhirR1CSScheme::new_for_r1cs with w1_size (r1cs-compiler/src/whir_r1cs.rs:48-92):
 * m = max(ceil log2 w1_size, ceil log2 (num_witnesses - w1_size), 13), plus
 * one when fewer than 4 m0 entries of w1's padding are free; m0 as in
 * pkg_r1cs_sizing.  w1_size = num_witnesses gives pkg_r1cs_sizing. */
int pkg_r1cs_sizing_split(size_t num_constraints, size_t num_witnesses, size_t w1_size,
                          size_t *m, size_t *m0);
/* r1cs: device arrays as for pkg_prove_r1cs; the struct is copied, the
 * arrays it points to must stay valid until finish returns.  w1: device,
 * w1_size Fr (16-byte aligned), copied.  Requires num_public_inputs + 1 <=
 * w1_size <= num_witnesses and every offset < 2^m.  Outputs (host):
 * whir_commit_words1 (pkg_whir_commit_words), challenges (num_challenges
 * Fr, Montgomery form: the values w2 holds at the offsets), *state.
 * Synchronous; device memory for both commitments is held until free. */
int pkg_dual_prove_begin(const pkg_r1cs *r1cs, size_t w1_size, const size_t *challenge_offsets,
                         size_t num_challenges, const uint64_t *w1, uint64_t blinding_seed,
                         uint64_t transcript_domain, const pkg_whir_params *whir,
                         uint64_t *whir_commit_words1, uint64_t *challenges,
                         pkg_dual_prove **state, pkg_stream_t stream);
/* w2: device, num_witnesses - w1_size Fr (16-byte aligned; NULL when
 * empty).  Outputs (host): out, whir_commit_words2, whir_proof1
 * (pkg_whir_proof_words(whir, 4 + (public inputs > 0)) words), whir_proof2
 * (pkg_whir_proof_words(whir, 3 + (num_challenges > 0))).  Once per state;
 * on the stream given to begin.  Synchronous. */
int pkg_dual_prove_finish(pkg_dual_prove *state, const uint64_t *w2, pkg_dual_proof *out,
                          uint64_t *whir_commit_words2, uint64_t *whir_proof1,
                          uint64_t *whir_proof2);
void pkg_dual_prove_free(pkg_dual_prove *state);

/* ---- Prover handles (tooling/provekit-ffi/src/ffi.rs, types.rs) ----------
 * The reference's FFI hands out an opaque PKProver (a prepared circuit) and
 * returns proofs in a PKBuf that the library allocated and pk_free_buf
 * releases.  Same conventions here, over the device prover: the handle holds
 * the circuit resident on the device that was current at creation, with its
 * transposes built once; a proof comes back in a pkg_buf.  Calls on one
 * handle are serialised (one proof at a time, synchronous); different
 * handles prove concurrently.  Statuses are this header's PKG_* codes; the
 * reference's PKStatus values are positive, and map as PKG_OK = PK_SUCCESS,
 * PKG_ERR_INVALID_ARGUMENT = InvalidInput or SchemeReadError, the other
 * PKG_ERR_* codes = ProofError. */
/* PKBuf (tooling/provekit-ffi/src/types.rs:8-40, include/provekit_ffi.h:14-22):
 * library-allocated bytes, released exactly once by pkg_free_buf. */
typedef struct {
  uint8_t *ptr;
  size_t len;
  size_t cap;
} pkg_buf;
/* pk_free_buf (ffi.rs:744-750); an empty buffer (ptr NULL) is a no-op. */
void pkg_free_buf(pkg_buf buf);
/* pk_get_last_error (ffi.rs:73-89): the calling thread's last message as
 * UTF-8 bytes (empty buffer if none), then cleared; free with pkg_free_buf. */
int pkg_get_last_error(pkg_buf *out);
/* pk_init (ffi.rs:92-97): checks that a CUDA device is present.  Optional
 * (every entry point initialises what it needs on first use). */
int pkg_init(void);

typedef struct pkg_prover pkg_prover;  /* PKProver (types.rs) */
typedef struct {
  unsigned folding_factor;   /* WHIR folding factor (reference default 3)   */
  unsigned log_inv_rate;     /* starting rate 2^-log_inv_rate (default 2)   */
  unsigned security_bits;    /* default 128                                 */
  unsigned pow_bits;         /* default 10                                  */
  int zk;                    /* 1: whir-ZK, the witness committed with a    */
                             /* blinding polynomial (WhirZkConfig, default) */
  uint64_t transcript_domain;/* Fiat-Shamir domain separator               */
} pkg_prover_config;
/* The reference's configuration (provekit/r1cs-compiler/src/whir_r1cs.rs:94-117). */
int pkg_prover_config_default(pkg_prover_config *cfg);
/* A prepared prover from an R1CS in host memory (CSR A, B, C over
 * num_witnesses columns, one Fr per nonzero, Montgomery form; witness[1 ..=
 * num_public_inputs] are public).  Replaces pk_prepare / pk_load_prover
 * (ffi.rs:160-265) as far as the prover goes: the reference compiles a Noir
 * circuit or reads a .pkp file, which is outside this library (Noir
 * compilation and the .pkp serde layout of the un-vendored whir / spongefish
 * types).  Row pointers, column indices and coefficients (canonical field
 * elements, below p) are validated on the host.  Synchronous; the handle is
 * freed by pkg_prover_free. */
int pkg_prover_create(size_t num_constraints, size_t num_witnesses, size_t num_public_inputs,
                      const uint64_t *const row_ptr[3], const uint32_t *const cols[3],
                      const uint64_t *const vals[3], const size_t nnz[3],
                      const pkg_prover_config *cfg, pkg_prover **out);
/* pk_free_prover (ffi.rs:703-718); NULL is a no-op. */
void pkg_prover_free(pkg_prover *prover);
typedef struct {
  size_t num_constraints, num_witnesses, num_public_inputs;
  size_t m, m0;              /* committed and sumcheck variables            */
  size_t num_statements;     /* WHIR statements: 4, or 5 with public inputs */
  size_t proof_bytes;        /* length of every proof this handle returns   */
  int device;
  pkg_whir_params whir;
} pkg_prover_info;
int pkg_prover_get_info(const pkg_prover *prover, pkg_prover_info *info);
/* A whole proof (pkg_prove_r1cs) of a solved witness: num_witnesses Fr in
 * host memory (Montgomery form).  Replaces pk_prove_json / pk_prove_toml
 * (ffi.rs:537-666), whose input maps go through Noir's witness solver first.
 * out_proof receives a library-owned buffer (pkg_free_buf) in this layout,
 * all integers little-endian:
 *   "PKGPROOF", u32 version (1), u32 0,
 *   u64 m, m0, num_public_inputs, num_statements, commit_words, proof_words,
 *       transcript_domain,
 *   the WHIR parameters as a pkg_whir_params struct: 104 bytes,
 *   root (32 bytes), then Fr (4 u64 each): r[m0], round coefficients[4 m0],
 *   alpha[m0], rho, sum_g, blinding_eval, public_x, evals[3], public_hash
 *   (canonical), public_eval, the transcript state before the WHIR proof (l,
 *   r; a verifier recomputes it),
 *   commit_words u64 (root, OOD answers), proof_words u64 (the WHIR proof).
 * The reference's .np layout (header + postcard + zstd over whir's and
 * spongefish's proof types) cannot be produced without those crates. */
int pkg_prover_prove(pkg_prover *prover, const uint64_t *witness, uint64_t blinding_seed,
                     pkg_buf *out_proof);
/* pk_serialize_prover / pk_load_prover_bytes (ffi.rs:329-362, 455-482) over
 * this library's own layout: "PKGPROVR", u32 version (1), u32 0, u64
 * num_constraints, num_witnesses, num_public_inputs, nnz[3], u32
 * folding_factor, log_inv_rate, security_bits, pow_bits, zk, 0, u64
 * transcript_domain, u64 0, then per matrix row_ptr (u64 x
 * num_constraints + 1), cols (u32 x nnz, zero-padded to 8 bytes), vals (Fr x
 * nnz).  Loading validates every size against the input length and the
 * matrices as pkg_prover_create does. */
int pkg_prover_serialize(const pkg_prover *prover, pkg_buf *out);
int pkg_prover_load_bytes(const uint8_t *ptr, size_t len, pkg_prover **out);

/* ---- field arithmetic (skyscraper/bn254-multiplier/src/scalar.rs:12-132,
 *      ark-ff Montgomery conversion) ---------------------------------------- */
/* out[i] = op(a[i], b[i]) over n Fr (4 x u64 LE each, device, 16-byte
 * aligned), asynchronous on stream; results fully reduced (< p).
 *   PKG_FR_MUL_F64 / PKG_FR_SQR_F64: a*b*2^-256, a^2*2^-256 mod p on the FP64
 *     pipe (the routines of the NTT and Skyscraper kernels); inputs < 2p.
 *   PKG_FR_FROM_MONT_F64: a*2^-256 mod p on the FP64 pipe; any 256-bit a.
 *   PKG_FR_MUL_INT / PKG_FR_SQR_INT: the same on the integer pipe; inputs < p.
 *   PKG_FR_FROM_MONT_INT: the same on the integer pipe (REDC alone); any 256-bit a.
 * b is read only by the two products (may be NULL otherwise).  The reference's
 * scalar_mul/scalar_sqr return values in [0, 2^256 - 2p) with the same
 * residue; only the residue is part of the contract. */
#define PKG_FR_MUL_F64 0
#define PKG_FR_SQR_F64 1
#define PKG_FR_FROM_MONT_F64 2
#define PKG_FR_MUL_INT 3
#define PKG_FR_SQR_INT 4
#define PKG_FR_FROM_MONT_INT 5
int pkg_fr_mul_batch(const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n, int op,
                     pkg_stream_t stream);

/* ---- memory ------------------------------------------------------------------ */
/* Device scratch (prove, sumcheck, transposes, server requests) comes from a
 * stream-ordered pool private to this library on each device, which keeps
 * the memory it has grown to so that repeated proofs do not map it again.
 * Returns unused pool memory on the current device to the driver, keeping at
 * least keep_bytes.  No counterpart in the reference. */
int pkg_trim_memory(size_t keep_bytes);
/* Indexed Fr sampler on the device (no rejection, every element computed
 * alone): out[i] = lo + hi 2^253 mod p (Montgomery form), lo and hi the two
 * 32-byte halves of ChaCha20 block start + i (RFC 8439 block function, key =
 * seed LE, nonce word 1), each read as a little-endian integer masked to 253
 * bits.  Draws the WHIR-ZK blinding polynomial of pkg_prove_r1cs.  out:
 * device, 16-byte aligned; async.  No counterpart in the reference (which
 * draws masks from thread_rng). */
int pkg_sample_fr_indexed(uint64_t seed, uint64_t start, size_t n, uint64_t *out,
                          pkg_stream_t stream);
/* Grows the pool on the current device to hold at least `bytes` more (one
 * allocation, freed and waited for).  The pool hands a block freed on one
 * stream to another stream only once its free has completed, so work on
 * several streams at once (proofs on their own streams, server workers)
 * otherwise grows the pool while it runs; reserving first keeps those
 * physical mappings out of the timed work.  No counterpart in the
 * reference. */
int pkg_reserve_memory(size_t bytes);

/* A host thread that proves keeps a few small resources for its later calls:
 * a mapped pinned buffer for reduction results (2 KiB), a pinned bounce
 * buffer for small reads (256 KiB), and per device a ~60 KiB device block
 * (reduction counter, partials, PoW word) and a grow-only pinned staging
 * buffer for a proof's STIR openings (about 0.3 MB at 2^20 constraints).
 * They are released when the thread exits; this releases the calling
 * thread's now (they are re-created on its next call).  The thread must have
 * no work of this library in flight.  No counterpart in the reference. */
int pkg_release_thread_resources(void);
/* Bytes those per-thread resources hold over all live threads: pinned host
 * memory and device memory.  Diagnostics; no counterpart in the reference. */
int pkg_thread_resource_bytes(size_t *host_bytes, size_t *device_bytes);

/* ---- diagnostics ---------------------------------------------------------- */
/* Synchronous device -> host copy of library-owned memory (e.g. batch buffers). */
int pkg_copy_to_host(void *dst, const void *src, size_t bytes);
/* Number of kernels this library has launched in this process. */
uint64_t pkg_kernel_launches(void);
/* Measured 32-bit IMAD-class throughput of the current device (instructions
 * per second, from a dependent-chain-free mad.lo/madc.hi microbenchmark).
 * Synchronous. */
int pkg_measure_imad_rate(double *instr_per_second);

/* Sustained double-precision fma rate of this GPU (fma instructions per
 * second, one thread-instruction each), from eight independent chains per
 * thread on every SM.  Denominator of the FP64-pipe roofline: the Fr
 * products of the NTT butterflies and Skyscraper rounds run on that pipe.
 * Synchronous.  No counterpart in the reference (a measurement helper). */
int pkg_measure_dfma_rate(double *instr_per_second);

#ifdef __cplusplus
}
#endif
#endif
