// internal.cuh -- device-side entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/provekit_b200.h"

namespace pk {

int merkle_tree_fr_device(const uint64_t* cw, size_t fr_per_leaf, size_t num_leaves, int encoding,
                          uint8_t* layers, cudaStream_t s);
// a = A w, b = B w, c = a o b over the R1CS's rows, zero-padded to padded
// entries (calculate_witness_bounds), one launch; err: device word, zeroed.
int witness_bounds_device(const pkg_r1cs* r1cs, const uint64_t* w, size_t padded, uint64_t* ta,
                          uint64_t* tb, uint64_t* tc, uint32_t* err, cudaStream_t s);
// y = M x for a CSR matrix; err: device word, zeroed; nnz: row_ptr[num_rows]
// if known (large matrices then take two balanced passes), else 0.
int spmv_device(const uint64_t* row_ptr, const uint32_t* cols, const uint64_t* vals,
                size_t num_rows, size_t num_cols, const uint64_t* x, uint64_t* y, uint32_t* err,
                cudaStream_t s, size_t nnz);
// eq(r, .) over the first num_entries points; sync: wait for the copy of r
int eq_hypercube_device(const uint64_t* r_host, size_t nr, size_t num_entries, uint64_t* out,
                        cudaStream_t s, bool sync = true);
// Skyscraper PoW on stream s (synchronous): generic::solve's answer.
int pow_solve_device(const uint64_t challenge[4], const uint64_t threshold[4], cudaStream_t s,
                     uint64_t* nonce_out);
// w += sum_j coeffs_j eq(points_j, .) (pkg_eq_accumulate); sync = false only
// when points and coeffs are pageable host memory.  expanded: points holds
// npts x nv coordinates; otherwise npts univariate points z, expanded on the
// device to (z^(2^(nv-1)), .., z^2, z).
int eq_accumulate_device(uint64_t* w, size_t nv, const uint64_t* points, const uint64_t* coeffs,
                         size_t npts, cudaStream_t s, bool sync, bool expanded = true);
// Codeword rows and their Merkle paths for nq indices (host in/out), one sync.
// sync = false: rows and paths are pinned host memory that the copies fill
// in stream order, and the caller synchronises before reading them.
int open_rows_device(const uint64_t* codeword, size_t fr_per_row, size_t num_rows,
                     const uint8_t* layers, const uint64_t* indices, size_t nq, uint64_t* rows,
                     uint8_t* paths, cudaStream_t s, bool sync = true);
// <a, b> to out, a slot of the thread's fused slots (FusedSlots: out within
// dev, ticket its ticket), in one launch; part: red_grid(n) Fr of scratch.
int dot_device(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out, uint64_t* part,
               cudaStream_t s, unsigned* ticket);

// The WHIR prover's round loop (pkg_whir_prove); values (host, ncov Fr) are
// the statements' values when the caller already has them, else nullptr;
// hat (device, 2^n Fr, overwritten) is zeta(coeffs) when the caller already
// computed it, else nullptr.
int whir_prove_device(const pkg_whir_params* p, pkg_transcript* t, const uint64_t* coeffs,
                      const uint64_t* codeword, const uint8_t* layers, const uint64_t* ood_points,
                      const uint64_t* covectors, size_t ncov, const uint64_t* values,
                      uint64_t* hat, uint64_t* proof, cudaStream_t s);
// In place v[b | 2^i] += v[b] over 2^n entries (pkg_subset_transform's zeta).
int subset_zeta_device(uint64_t* v, unsigned n, cudaStream_t s);

// ---- the R1CS prove paths (prove.cu, dual_prove.cu) -----------------------
// Seeds of the whir-ZK mask polynomials: the blinding seed with the first
// and the second 64 fraction bits of pi (fixed, arbitrary separators), the
// first for the (first) witness commitment, the second for w2's.
constexpr uint64_t kMaskSeed = 0x243f6a8885a308d3ULL;
constexpr uint64_t kMaskSeed2 = 0x13198a2e03707344ULL;
// get_public_weights (provekit/prover/src/whir_r1cs.rs:665-676): w[0 ..= np]
// read from the device witness into pubw (host, 4 (np + 1) words), the
// hash of w[1 ..= np] (PublicInputs::hash, common/src/witness/mod.rs:86-97;
// canonical, 0 without public inputs) absorbed, the challenge x squeezed.
int public_challenge(const uint64_t* witness, size_t np, uint64_t* pubw, pkg_transcript* t,
                     uint64_t hash[4], uint64_t x[4], cudaStream_t s);
// make_public_weight's entries [1, x, .., x^np] (prefix_covector.rs:173-186)
// into xpow (4 (np + 1) words) and <xpow, pubw> into eval (Montgomery form).
void public_weight_host(const uint64_t* pubw, size_t np, const uint64_t x[4], uint64_t* xpow,
                        uint64_t eval[4]);
// The blinding covector expand_powers::<4>(alpha) (whir_r1cs.rs:184):
// [1, a_i, a_i^2, a_i^3] for each of the m0 challenges; bw: 16 m0 words.
void blinding_weights_host(const uint64_t* alpha, size_t m0, uint64_t* bw);

}  // namespace pk
