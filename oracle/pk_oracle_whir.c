/*
 * pk_oracle_whir.c -- CPU restatement of a whole WHIR proof: the round
 * orchestration around the building blocks of pk_oracle.c.
 *
 * TEST INFRASTRUCTURE ONLY (see pk_oracle.h): the parity oracle for the
 * device prover pkg_whir_prove, and the verifier its proofs are checked with.
 *
 * The whir crate (prover and verifier) is not vendored with the reference.
 * The round structure restated here is the one the reference's Go verifier
 * walks (runWhir, recursive-verifier/app/circuit/whir.go:587-724):
 *   commitment: root, OOD points and answers;
 *   statement evaluations, combination randomness, initial sumcheck of k
 *   rounds (runWhirSumcheckRounds, circuit/whir_utilities.go:103-126);
 *   per round: root of the folded polynomial's codeword, OOD, PoW
 *   (RunPoW, whir.go:726-735), STIR indices on the previous codeword
 *   (getStirChallenges, whir_utilities.go:49-78) with Merkle openings
 *   (verifyMerkleTreeProofs, :14-47) folded by computeFold (:182-188),
 *   combination randomness (GenerateCombinationRandomness, whir.go:770-778),
 *   the claimed sum shifted by calculateShiftValue (:190-192), k sumcheck
 *   rounds;
 *   final: the remaining polynomial's coefficients, PoW, STIR queries whose
 *   folds must equal UnivarPoly of those coefficients, the final sumcheck,
 *   and lastEval == W(r) * f(r) (computeWPoly, whir_utilities.go:128-161).
 * Conventions that the un-vendored crate fixes and that are chosen here are
 * listed in pk_oracle.h beside pko_whir_params.
 */
#include "pk_oracle.h"

#include <stdlib.h>
#include <string.h>

static const uint64_t PMOD[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                                 0xb85045b68181585dULL, 0x30644e72e131a029ULL};
static const uint64_t ONE_M[4] = {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL,
                                  0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL};

static void cp4(uint64_t *d, const uint64_t *s) { memcpy(d, s, 32); }
static int is_canon(const uint64_t a[4]) {
    for (int i = 3; i >= 0; i--)
        if (a[i] != PMOD[i]) return a[i] < PMOD[i];
    return 0;
}
static int eq4(const uint64_t *a, const uint64_t *b) { return memcmp(a, b, 32) == 0; }
static void mont_u64(uint64_t r[4], uint64_t v) {
    uint64_t c[4] = {v, 0, 0, 0};
    pko_fr_to_mont(r, c);
}

/* ---- parameters ---------------------------------------------------------- */
static unsigned rows_log(const pko_whir_params *p, unsigned r) {
    return p->num_variables + p->log_inv_rate - p->folding_factor - r;
}

static int params_ok(const pko_whir_params *p) {
    if (!p) return 0;
    unsigned n = p->num_variables, k = p->folding_factor, R = p->num_rounds;
    if (k < 1 || k > 6 || n > 30 || R > PKO_WHIR_MAX_ROUNDS) return 0;
    if (p->log_inv_rate < 1 || p->log_inv_rate > 8) return 0;
    if ((R + 1) * k + p->final_vars != n) return 0;
    if (p->ood_samples > 4 || p->pow_bits > 27 || p->final_pow_bits > 27) return 0;
    if (p->batch_size != 1 && p->batch_size != 2 && p->batch_size != 4) return 0;
    if (n + p->log_inv_rate < k + R + 1) return 0; /* every codeword has >= 2 rows */
    for (unsigned r = 0; r <= R; r++)
        if (p->queries[r] < 1 || p->queries[r] > 4096) return 0;
    return 1;
}

int pko_whir_params_init(pko_whir_params *p, unsigned n, unsigned k, unsigned log_inv_rate,
                         unsigned security_bits, unsigned pow_bits) {
    if (!p || k < 1 || k > 6 || n < k || n > 30 || log_inv_rate < 1 || log_inv_rate > 8 ||
        pow_bits > 27 || security_bits <= pow_bits || security_bits > 512)
        return PKO_WHIR_BAD_PARAMS;
    memset(p, 0, sizeof *p);
    unsigned folds = n > 6 ? (n - 6 + k - 1) / k : 1;
    if (folds * k > n) folds = n / k;
    if (folds < 1 || folds - 1 > PKO_WHIR_MAX_ROUNDS) return PKO_WHIR_BAD_PARAMS;
    p->num_variables = n;
    p->folding_factor = k;
    p->log_inv_rate = log_inv_rate;
    p->num_rounds = folds - 1;
    p->final_vars = n - folds * k;
    p->ood_samples = 1;
    p->pow_bits = pow_bits;
    p->final_pow_bits = pow_bits;
    p->batch_size = 1;
    for (unsigned r = 0; r <= p->num_rounds; r++) {
        unsigned rate = log_inv_rate + r * (k - 1);
        unsigned q = (2 * (security_bits - pow_bits) + rate - 1) / rate;
        p->queries[r] = q > 4096 ? 4096 : q;
    }
    return params_ok(p) ? 0 : PKO_WHIR_BAD_PARAMS;
}

size_t pko_whir_commit_words(const pko_whir_params *p) {
    return 4 + 4 * (size_t)p->ood_samples * p->batch_size;
}

/* Fr per opened row of codeword r: the first codeword holds every batched
 * polynomial's values. */
static size_t row_fr(const pko_whir_params *p, unsigned r) {
    return ((size_t)1 << p->folding_factor) * (r == 0 ? p->batch_size : 1);
}

size_t pko_whir_proof_words(const pko_whir_params *p, size_t ncov) {
    if (!params_ok(p)) return 0;
    const size_t k = p->folding_factor;
    size_t w = 4 * ncov * p->batch_size + 12 * k;
    for (unsigned r = 0; r < p->num_rounds; r++)
        w += 4 + 4 * (size_t)p->ood_samples + (p->pow_bits ? 1 : 0) +
             (size_t)p->queries[r] * (4 * row_fr(p, r) + 4 * rows_log(p, r)) + 12 * k;
    const unsigned R = p->num_rounds;
    w += 4 * ((size_t)1 << p->final_vars) + (p->final_pow_bits ? 1 : 0) +
         (size_t)p->queries[R] * (4 * row_fr(p, R) + 4 * rows_log(p, R)) +
         12 * (size_t)p->final_vars;
    return w;
}

/* ---- transcript bytes, transforms, commitment ---------------------------- */
void pko_transcript_squeeze_bytes(pko_transcript *t, uint8_t *out, size_t n) {
    size_t done = 0;
    while (done < n) {
        uint64_t m[4], c[4];
        uint8_t b[32];
        pko_transcript_squeeze(t, m);
        pko_fr_from_mont(c, m);
        for (int i = 0; i < 32; i++) b[i] = (uint8_t)(c[i / 8] >> (8 * (i % 8)));
        size_t take = n - done < 31 ? n - done : 31;
        memcpy(out + done, b, take);
        done += take;
    }
}

void pko_subset_zeta(uint64_t *v, unsigned n) {
    const size_t N = (size_t)1 << n;
    for (unsigned i = 0; i < n; i++) {
        const size_t h = (size_t)1 << i;
#pragma omp parallel for schedule(static)
        for (size_t b = 0; b < N; b++)
            if (b & h) pko_fr_add(v + 4 * b, v + 4 * b, v + 4 * (b ^ h));
    }
}

void pko_subset_mobius_t(uint64_t *v, unsigned n) {
    const size_t N = (size_t)1 << n;
    for (unsigned i = 0; i < n; i++) {
        const size_t h = (size_t)1 << i;
#pragma omp parallel for schedule(static)
        for (size_t b = 0; b < N; b++)
            if (!(b & h)) pko_fr_sub(v + 4 * b, v + 4 * b, v + 4 * (b | h));
    }
}

int pko_whir_commit(const uint64_t *coeffs, size_t num_coeffs, unsigned k, unsigned log_inv_rate,
                    uint64_t *codeword, uint8_t *layers) {
    const size_t M = (size_t)1 << k;
    if (k > 12 || !num_coeffs || (num_coeffs & (num_coeffs - 1)) || num_coeffs < M) return -1;
    const size_t len = num_coeffs / M, L = len << log_inv_rate;
    int rc = pko_rs_interleaved_encode(coeffs, M, len, NULL, 0, L, codeword);
    if (rc) return rc;
    uint64_t *canon = (uint64_t *)malloc(32 * L * M);
    if (!canon) return -2;
    memcpy(canon, codeword, 32 * L * M);
    pko_from_mont_many(canon, L * M);
    rc = pko_merkle_tree((const uint8_t *)canon, 32 * M, L, layers);
    free(canon);
    return rc;
}

/* ---- shared protocol pieces --------------------------------------------- */
static void powers(uint64_t *out, const uint64_t base[4], size_t n) {
    if (n) cp4(out, ONE_M);
    for (size_t i = 1; i < n; i++) pko_fr_mul(out + 4 * i, out + 4 * (i - 1), base);
}

static void pow_threshold(uint64_t thr[4], unsigned bits) {
    cp4(thr, PMOD);
    for (unsigned s = 0; s < bits; s++) {
        thr[0] = (thr[0] >> 1) | (thr[1] << 63);
        thr[1] = (thr[1] >> 1) | (thr[2] << 63);
        thr[2] = (thr[2] >> 1) | (thr[3] << 63);
        thr[3] >>= 1;
    }
}

static int less4(const uint64_t a[4], const uint64_t b[4]) {
    for (int i = 3; i >= 0; i--)
        if (a[i] != b[i]) return a[i] < b[i];
    return 0;
}

static void reverse_fr(uint64_t *out, const uint64_t *in, size_t n) {
    for (size_t i = 0; i < n; i++) cp4(out + 4 * i, in + 4 * (n - 1 - i));
}

/* t[i] += r (t[i + size/2] - t[i]) for the two tables: bind the top variable. */
static void fold_tables(uint64_t *E, uint64_t *w, size_t size, const uint64_t r[4]) {
    const size_t h = size / 2;
    uint64_t *tabs[2] = {E, w};
    for (int j = 0; j < 2; j++) {
        uint64_t *t = tabs[j];
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < h; i++) {
            uint64_t d[4];
            pko_fr_sub(d, t + 4 * (i + h), t + 4 * i);
            pko_fr_mul(d, d, r);
            pko_fr_add(t + 4 * i, t + 4 * i, d);
        }
    }
}

/* EvaluateQuadraticPolynomialFromEvaluationList (utilities/utilities.go:149-155). */
static void quad_eval(uint64_t out[4], const uint64_t h[12], const uint64_t x[4]) {
    uint64_t two[4], inv2[4], t[4], b1[4], b2[4];
    pko_fr_add(two, ONE_M, ONE_M);
    pko_fr_inv(inv2, two);
    /* b1 = (-h2 + 4 h1 - 3 h0) / 2 */
    pko_fr_add(t, h + 4, h + 4);
    pko_fr_add(t, t, t);
    pko_fr_sub(t, t, h + 8);
    pko_fr_sub(t, t, h);
    pko_fr_sub(t, t, h);
    pko_fr_sub(t, t, h);
    pko_fr_mul(b1, t, inv2);
    /* b2 = (h2 - 2 h1 + h0) / 2 */
    pko_fr_sub(t, h + 8, h + 4);
    pko_fr_sub(t, t, h + 4);
    pko_fr_add(t, t, h);
    pko_fr_mul(b2, t, inv2);
    /* b2 x^2 + b1 x + h0 */
    pko_fr_mul(t, b2, x);
    pko_fr_add(t, t, b1);
    pko_fr_mul(t, t, x);
    pko_fr_add(out, t, h);
}

/* EqPolyOutside (utilities.go:141-147) of ExpandFromUnivariate(z, m) and r. */
static void eq_expand(uint64_t out[4], const uint64_t z[4], const uint64_t *r, size_t m) {
    uint64_t *e = (uint64_t *)malloc(32 * (m ? m : 1));
    uint64_t acc[4], a[4], b[4], one_e[4], one_r[4];
    pko_expand_from_univariate(e, z, m);
    cp4(acc, ONE_M);
    for (size_t i = 0; i < m; i++) {
        pko_fr_mul(a, e + 4 * i, r + 4 * i);
        pko_fr_sub(one_e, ONE_M, e + 4 * i);
        pko_fr_sub(one_r, ONE_M, r + 4 * i);
        pko_fr_mul(b, one_e, one_r);
        pko_fr_add(a, a, b);
        pko_fr_mul(acc, acc, a);
    }
    cp4(out, acc);
    free(e);
}

/* ---- prover -------------------------------------------------------------- */
typedef struct {
    uint64_t *p;
    size_t pos;
} cursor;

static void put4(cursor *c, const uint64_t *x) {
    cp4(c->p + c->pos, x);
    c->pos += 4;
}

static int sc_prove(pko_transcript *t, uint64_t *E, uint64_t *w, size_t *size, unsigned rounds,
                    uint64_t *rands, cursor *c) {
    for (unsigned i = 0; i < rounds; i++) {
        uint64_t h[12];
        int rc = pko_whir_sumcheck_round(E, w, *size, NULL, h);
        if (rc) return rc;
        memcpy(c->p + c->pos, h, 96);
        c->pos += 12;
        for (int j = 0; j < 3; j++) pko_transcript_absorb(t, h + 4 * j);
        pko_transcript_squeeze(t, rands + 4 * i);
        fold_tables(E, w, *size, rands + 4 * i);
        *size /= 2;
    }
    return 0;
}

static void pow_prove(pko_transcript *t, unsigned bits, cursor *c) {
    uint64_t cm[4], ch[4], thr[4], nm[4];
    pko_transcript_squeeze(t, cm);
    pko_fr_from_mont(ch, cm);
    pow_threshold(thr, bits);
    uint64_t nonce = pko_sky_pow_solve(ch, thr);
    c->p[c->pos++] = nonce;
    mont_u64(nm, nonce);
    pko_transcript_absorb(t, nm);
}

static int stir_indices_from(pko_transcript *t, size_t q, size_t L, uint64_t *idx) {
    int bits = 0;
    while (((size_t)1 << bits) < L) bits++;
    const size_t nb = (size_t)(bits + 7) / 8;
    uint8_t *bytes = (uint8_t *)malloc(q * nb + 1);
    if (!bytes) return -2;
    pko_transcript_squeeze_bytes(t, bytes, q * nb);
    pko_stir_indices(bytes, L, q, idx);
    free(bytes);
    return bits;
}

static int stir_prove(pko_transcript *t, size_t q, size_t L, size_t K, const uint64_t *cw,
                      const uint8_t *layers, uint64_t *idx, cursor *c) {
    /* K: Fr per row (the batch's width for the first codeword) */
    int depth = stir_indices_from(t, q, L, idx);
    if (depth < 0) return depth;
    for (size_t i = 0; i < q; i++) {
        memcpy(c->p + c->pos, cw + 4 * K * idx[i], 32 * K);
        c->pos += 4 * K;
        int rc = pko_merkle_open(layers, L, idx[i], (uint8_t *)(c->p + c->pos));
        if (rc) return rc;
        c->pos += 4 * (size_t)depth;
    }
    return 0;
}

int pko_whir_commit_ood(const pko_whir_params *p, pko_transcript *t, const uint64_t *coeffs,
                        const uint8_t root[32], uint64_t *commit_words, uint64_t *ood_points) {
    if (!params_ok(p)) return PKO_WHIR_BAD_PARAMS;
    uint64_t rc[4], rm[4];
    memcpy(rc, root, 32);
    if (!is_canon(rc)) return PKO_WHIR_BAD_PARAMS;
    pko_fr_to_mont(rm, rc);
    pko_transcript_absorb(t, rm);
    cp4(commit_words, rc);
    const size_t N = (size_t)1 << p->num_variables;
    const unsigned o = p->ood_samples;
    for (unsigned j = 0; j < o; j++) pko_transcript_squeeze(t, ood_points + 4 * j);
    for (unsigned i = 0; i < p->batch_size; i++)
        for (unsigned j = 0; j < o; j++) {
            uint64_t *ans = commit_words + 4 + 4 * (i * o + j);
            pko_poly_eval(ans, coeffs + 4 * N * i, N, ood_points + 4 * j);
            pko_transcript_absorb(t, ans);
        }
    if (p->batch_size > 1) pko_transcript_squeeze(t, ood_points + 4 * o);
    return 0;
}

int pko_whir_prove(const pko_whir_params *p, pko_transcript *t, const uint64_t *coeffs,
                   const uint64_t *codeword, const uint8_t *layers, const uint64_t *commit_words,
                   const uint64_t *ood_points, const uint64_t *covectors, size_t ncov,
                   uint64_t *proof) {
    if (!params_ok(p) || ncov > 16) return PKO_WHIR_BAD_PARAMS;
    const unsigned n = p->num_variables, k = p->folding_factor, R = p->num_rounds;
    const unsigned o = p->ood_samples;
    const size_t N = (size_t)1 << n, K = (size_t)1 << k;
    int rc = 0;
    uint64_t *E = (uint64_t *)malloc(32 * N), *w = (uint64_t *)calloc(N, 32);
    uint64_t *f = (uint64_t *)malloc(32 * N), *g = (uint64_t *)malloc(32 * N);
    uint64_t *pw = (uint64_t *)malloc(32 * (o + ncov + 4096));
    uint64_t *pts = (uint64_t *)malloc(32 * (size_t)(n ? n : 1) * (o + 4096));
    uint64_t *upts = (uint64_t *)malloc(32 * (o + 4096));
    uint64_t *idx = (uint64_t *)malloc(8 * 4096);
    uint64_t alpha[6 * 4], ralpha[6 * 4], gamma[4];
    uint64_t *cw_own = NULL, *cw_next = NULL;
    uint8_t *lay_own = NULL, *lay_next = NULL;
    cursor c = {proof, 0};
    (void)commit_words;
    if (!E || !w || !f || !g || !pw || !pts || !upts || !idx) {
        rc = -2;
        goto done;
    }
    /* the batch: c = sum_i b^i f_i (b drawn at the commitment) */
    const unsigned Bn = p->batch_size;
    uint64_t bp[4 * 4];
    powers(bp, ood_points + 4 * o, Bn);
    memset(f, 0, 32 * N);
    for (unsigned i = 0; i < Bn; i++)
        for (size_t b = 0; b < N; b++) {
            uint64_t x[4];
            pko_fr_mul(x, bp + 4 * i, coeffs + 4 * (N * i + b));
            pko_fr_add(f + 4 * b, f + 4 * b, x);
        }
    memcpy(E, f, 32 * N);
    pko_subset_zeta(E, n);

    /* statement values, polynomial by polynomial */
    for (unsigned i = 0; i < Bn; i++)
        for (size_t a = 0; a < ncov; a++) {
            pko_dot(proof + c.pos, covectors + 4 * N * a, coeffs + 4 * N * i, N);
            pko_transcript_absorb(t, proof + c.pos);
            c.pos += 4;
        }
    pko_transcript_squeeze(t, gamma);
    powers(pw, gamma, o + ncov);
    for (size_t a = 0; a < ncov; a++) {
        const uint64_t *av = covectors + 4 * N * a;
#pragma omp parallel for schedule(static)
        for (size_t b = 0; b < N; b++) {
            uint64_t x[4];
            pko_fr_mul(x, pw + 4 * (o + a), av + 4 * b);
            pko_fr_add(w + 4 * b, w + 4 * b, x);
        }
    }
    pko_subset_mobius_t(w, n);
    for (unsigned j = 0; j < o; j++) pko_expand_from_univariate(pts + 4 * n * j, ood_points + 4 * j, n);
    if ((rc = pko_eq_accumulate(w, n, pts, pw, o))) goto done;

    size_t size = N;
    if ((rc = sc_prove(t, E, w, &size, k, alpha, &c))) goto done;

    unsigned nv = n;
    const uint64_t *cw_r = codeword;
    const uint8_t *lay_r = layers;
    for (unsigned r = 0; r < R; r++) {
        reverse_fr(ralpha, alpha, k);
        if ((rc = pko_whir_fold_coeffs(f, (size_t)1 << nv, k, ralpha, g))) goto done;
        nv -= k;
        const size_t Ln = (size_t)1 << rows_log(p, r + 1);
        cw_next = (uint64_t *)malloc(32 * K * Ln);
        lay_next = (uint8_t *)malloc(32 * (2 * Ln - 1));
        if (!cw_next || !lay_next) {
            rc = -2;
            goto done;
        }
        if ((rc = pko_whir_commit(g, (size_t)1 << nv, k, p->log_inv_rate + (r + 1) * (k - 1),
                                  cw_next, lay_next)))
            goto done;
        uint64_t root[4], rm[4];
        memcpy(root, lay_next + 32 * (2 * Ln - 2), 32);
        put4(&c, root);
        pko_fr_to_mont(rm, root);
        pko_transcript_absorb(t, rm);
        for (unsigned j = 0; j < o; j++) pko_transcript_squeeze(t, upts + 4 * j);
        for (unsigned j = 0; j < o; j++) {
            pko_poly_eval(proof + c.pos, g, (size_t)1 << nv, upts + 4 * j);
            pko_transcript_absorb(t, proof + c.pos);
            c.pos += 4;
        }
        if (p->pow_bits) pow_prove(t, p->pow_bits, &c);
        const size_t Lr = (size_t)1 << rows_log(p, r), q = p->queries[r];
        if ((rc = stir_prove(t, q, Lr, row_fr(p, r), cw_r, lay_r, idx, &c))) goto done;
        pko_rs_evaluation_points(Lr, (const size_t *)idx, q, upts + 4 * o);
        pko_transcript_squeeze(t, gamma);
        powers(pw, gamma, o + q);
        for (size_t j = 0; j < o + q; j++) pko_expand_from_univariate(pts + 4 * nv * j, upts + 4 * j, nv);
        if ((rc = pko_eq_accumulate(w, nv, pts, pw, o + q))) goto done;
        if ((rc = sc_prove(t, E, w, &size, k, alpha, &c))) goto done;
        /* advance: f <- g, C_r <- C_{r+1} */
        uint64_t *tmp = f;
        f = g;
        g = tmp;
        free(cw_own);
        free(lay_own);
        cw_own = cw_next;
        lay_own = lay_next;
        cw_next = NULL;
        lay_next = NULL;
        cw_r = cw_own;
        lay_r = lay_own;
    }
    /* final polynomial, PoW, queries, sumcheck */
    reverse_fr(ralpha, alpha, k);
    if ((rc = pko_whir_fold_coeffs(f, (size_t)1 << nv, k, ralpha, g))) goto done;
    nv -= k;
    for (size_t i = 0; i < ((size_t)1 << nv); i++) {
        put4(&c, g + 4 * i);
        pko_transcript_absorb(t, g + 4 * i);
    }
    if (p->final_pow_bits) pow_prove(t, p->final_pow_bits, &c);
    if ((rc = stir_prove(t, p->queries[R], (size_t)1 << rows_log(p, R), row_fr(p, R), cw_r, lay_r,
                         idx, &c)))
        goto done;
    {
        uint64_t *rfin = (uint64_t *)malloc(32 * (nv ? nv : 1));
        rc = rfin ? sc_prove(t, E, w, &size, nv, rfin, &c) : -2;
        free(rfin);
        if (rc) goto done;
    }
    if (c.pos != pko_whir_proof_words(p, ncov)) rc = -3;
done:
    free(E);
    free(w);
    free(f);
    free(g);
    free(pw);
    free(pts);
    free(upts);
    free(idx);
    free(cw_own);
    free(lay_own);
    free(cw_next);
    free(lay_next);
    return rc;
}

/* ---- verifier ------------------------------------------------------------ */
typedef struct {
    const uint64_t *p;
    size_t pos, len;
    int bad;
} reader;

static const uint64_t *get_fr(reader *rd) {
    if (rd->pos + 4 > rd->len) {
        rd->bad = 1;
        return ONE_M;
    }
    const uint64_t *x = rd->p + rd->pos;
    rd->pos += 4;
    if (!is_canon(x)) rd->bad = 1;
    return x;
}

static uint64_t get_word(reader *rd) {
    if (rd->pos + 1 > rd->len) {
        rd->bad = 1;
        return 0;
    }
    return rd->p[rd->pos++];
}

static int sc_verify(pko_transcript *t, reader *rd, unsigned rounds, uint64_t last[4],
                     uint64_t *rands) {
    for (unsigned i = 0; i < rounds; i++) {
        uint64_t h[12], s[4];
        for (int j = 0; j < 3; j++) cp4(h + 4 * j, get_fr(rd));
        if (rd->bad) return PKO_WHIR_REJECT_FORMAT;
        for (int j = 0; j < 3; j++) pko_transcript_absorb(t, h + 4 * j);
        pko_transcript_squeeze(t, rands + 4 * i);
        pko_fr_add(s, h, h + 4); /* CheckSumOverBool (utilities.go:168-171) */
        if (!eq4(s, last)) return PKO_WHIR_REJECT_SUMCHECK;
        quad_eval(last, h, rands + 4 * i);
    }
    return 0;
}

static int pow_verify(pko_transcript *t, reader *rd, unsigned bits) {
    uint64_t cm[4], ch[4], thr[4], nm[4], h[4];
    pko_transcript_squeeze(t, cm);
    pko_fr_from_mont(ch, cm);
    uint64_t nonce = get_word(rd);
    if (rd->bad) return PKO_WHIR_REJECT_FORMAT;
    mont_u64(nm, nonce);
    pko_transcript_absorb(t, nm);
    pow_threshold(thr, bits);
    uint64_t nv[4] = {nonce, 0, 0, 0};
    pko_sky_compress(h, ch, nv);
    return less4(h, thr) ? 0 : PKO_WHIR_REJECT_POW;
}

/* Reads q openings of a codeword of L rows of `batch` polynomials, checks
 * them against root, collapses each row with the powers bp of the batching
 * challenge (rlcBatchedLeaves, mtUtilities.go:98-119) and writes the folds
 * (MultivarPoly with ralpha) and the evaluation points. */
static int stir_verify(pko_transcript *t, reader *rd, size_t q, size_t L, unsigned k,
                       unsigned batch, const uint64_t *bp, const uint64_t root[4],
                       const uint64_t *ralpha, uint64_t *folds, uint64_t *points) {
    const size_t K = (size_t)1 << k, W = K * batch;
    uint64_t *idx = (uint64_t *)malloc(8 * q);
    uint64_t *row = (uint64_t *)malloc(32 * W), *canon = (uint64_t *)malloc(32 * W);
    uint64_t col[64 * 4];
    int rc = 0;
    if (!idx || !row || !canon) {
        rc = -2;
        goto out;
    }
    int depth = stir_indices_from(t, q, L, idx);
    if (depth < 0) {
        rc = depth;
        goto out;
    }
    for (size_t i = 0; i < q; i++) {
        for (size_t j = 0; j < W; j++) cp4(row + 4 * j, get_fr(rd));
        if (rd->bad || rd->pos + 4 * (size_t)depth > rd->len) {
            rd->bad = 1;
            rc = PKO_WHIR_REJECT_FORMAT;
            goto out;
        }
        const uint8_t *path = (const uint8_t *)(rd->p + rd->pos);
        rd->pos += 4 * (size_t)depth;
        memcpy(canon, row, 32 * W);
        pko_from_mont_many(canon, W);
        if (!pko_merkle_verify(canon, W, idx[i], path, (size_t)depth, (const uint8_t *)root)) {
            rc = PKO_WHIR_REJECT_MERKLE;
            goto out;
        }
        for (size_t j = 0; j < K; j++) {
            uint64_t acc[4] = {0, 0, 0, 0}, x[4];
            for (unsigned b = 0; b < batch; b++) {
                pko_fr_mul(x, bp + 4 * b, row + 4 * (b * K + j));
                pko_fr_add(acc, acc, x);
            }
            cp4(col + 4 * j, acc);
        }
        pko_whir_fold_rows(col, 1, k, ralpha, folds + 4 * i);
    }
    pko_rs_evaluation_points(L, (const size_t *)idx, q, points);
out:
    free(idx);
    free(row);
    free(canon);
    return rc;
}

typedef struct {
    unsigned nv;
    size_t npts;
    uint64_t *pts, *coef;
} round_claims;

int pko_whir_verify_commit(const pko_whir_params *p, pko_transcript *t,
                           const uint64_t *commit_words, uint64_t *ood_points) {
    if (!params_ok(p)) return PKO_WHIR_BAD_PARAMS;
    uint64_t rm[4];
    if (!is_canon(commit_words)) return PKO_WHIR_REJECT_FORMAT;
    pko_fr_to_mont(rm, commit_words);
    pko_transcript_absorb(t, rm);
    for (unsigned j = 0; j < p->ood_samples; j++) pko_transcript_squeeze(t, ood_points + 4 * j);
    for (unsigned j = 0; j < p->ood_samples * p->batch_size; j++) {
        if (!is_canon(commit_words + 4 + 4 * j)) return PKO_WHIR_REJECT_FORMAT;
        pko_transcript_absorb(t, commit_words + 4 + 4 * j);
    }
    if (p->batch_size > 1) pko_transcript_squeeze(t, ood_points + 4 * p->ood_samples);
    return 0;
}

int pko_whir_verify(const pko_whir_params *p, pko_transcript *t, const uint64_t *covectors,
                    size_t ncov, const uint64_t *commit_words, const uint64_t *proof,
                    size_t proof_words) {
    uint64_t z[5 * 4];
    int rc = pko_whir_verify_commit(p, t, commit_words, z);
    if (rc) return rc;
    return pko_whir_verify_proof(p, t, covectors, ncov, commit_words, z, proof, proof_words);
}

int pko_whir_verify_proof(const pko_whir_params *p, pko_transcript *t, const uint64_t *covectors,
                          size_t ncov, const uint64_t *commit_words, const uint64_t *ood_points,
                          const uint64_t *proof, size_t proof_words) {
    if (!params_ok(p) || ncov > 16) return PKO_WHIR_BAD_PARAMS;
    if (proof_words != pko_whir_proof_words(p, ncov)) return PKO_WHIR_REJECT_FORMAT;
    const unsigned n = p->num_variables, k = p->folding_factor, R = p->num_rounds;
    const unsigned o = p->ood_samples, nf = p->final_vars;
    const size_t N = (size_t)1 << n;
    reader rd = {proof, 0, proof_words, 0};
    round_claims rounds[PKO_WHIR_MAX_ROUNDS];
    memset(rounds, 0, sizeof rounds);
    uint64_t *r_all = (uint64_t *)malloc(32 * (n ? n : 1));
    uint64_t *pw0 = (uint64_t *)malloc(32 * (o + ncov + 1));
    uint64_t *z0 = (uint64_t *)malloc(32 * (o + 1));
    uint64_t *folds = (uint64_t *)malloc(32 * 4096), *ypts = (uint64_t *)malloc(32 * 4096);
    uint64_t *fc = (uint64_t *)malloc(32 * ((size_t)1 << nf));
    uint64_t *lin = (uint64_t *)calloc(N, 32);
    uint64_t last[4] = {0, 0, 0, 0}, gamma[4], x[4], root[4], rm[4], ralpha[6 * 4];
    size_t nr = 0;
    int rc = 0;
    if (!r_all || !pw0 || !z0 || !folds || !ypts || !fc || !lin) {
        rc = -2;
        goto done;
    }
    /* the commitment's root and OOD points (pko_whir_verify_commit) */
    cp4(root, commit_words);
    if (o) memcpy(z0, ood_points, 32 * o);
    /* statement values (per polynomial) and the initial claimed sum over
     * the batch's combination c = sum_i b^i f_i */
    const unsigned Bn = p->batch_size;
    uint64_t bp[4 * 4], vals[16 * 4], cans[4 * 4];
    powers(bp, ood_points + 4 * o, Bn);
    memset(vals, 0, sizeof vals);
    memset(cans, 0, sizeof cans);
    for (unsigned i = 0; i < Bn; i++)
        for (size_t a = 0; a < ncov; a++) {
            uint64_t v[4];
            cp4(v, get_fr(&rd));
            if (rd.bad) {
                rc = PKO_WHIR_REJECT_FORMAT;
                goto done;
            }
            pko_transcript_absorb(t, v);
            pko_fr_mul(x, bp + 4 * i, v);
            pko_fr_add(vals + 4 * a, vals + 4 * a, x);
        }
    for (unsigned i = 0; i < Bn; i++)
        for (unsigned j = 0; j < o; j++) {
            pko_fr_mul(x, bp + 4 * i, commit_words + 4 + 4 * (i * o + j));
            pko_fr_add(cans + 4 * j, cans + 4 * j, x);
        }
    pko_transcript_squeeze(t, gamma);
    powers(pw0, gamma, o + ncov);
    for (unsigned j = 0; j < o; j++) {
        pko_fr_mul(x, pw0 + 4 * j, cans + 4 * j);
        pko_fr_add(last, last, x);
    }
    for (size_t a = 0; a < ncov; a++) {
        pko_fr_mul(x, pw0 + 4 * (o + a), vals + 4 * a);
        pko_fr_add(last, last, x);
    }
    if ((rc = sc_verify(t, &rd, k, last, r_all))) goto done;
    nr = k;
    for (unsigned r = 0; r < R; r++) {
        uint64_t prev_root[4];
        cp4(prev_root, root);
        cp4(root, get_fr(&rd));
        if (rd.bad) {
            rc = PKO_WHIR_REJECT_FORMAT;
            goto done;
        }
        pko_fr_to_mont(rm, root);
        pko_transcript_absorb(t, rm);
        const size_t q = p->queries[r];
        round_claims *rc_r = &rounds[r];
        rc_r->nv = n - (r + 1) * k;
        rc_r->npts = o + q;
        rc_r->pts = (uint64_t *)malloc(32 * (o + q));
        rc_r->coef = (uint64_t *)malloc(32 * (o + q));
        if (!rc_r->pts || !rc_r->coef) {
            rc = -2;
            goto done;
        }
        uint64_t ans[4 * 4];
        for (unsigned j = 0; j < o; j++) pko_transcript_squeeze(t, rc_r->pts + 4 * j);
        for (unsigned j = 0; j < o; j++) {
            cp4(ans + 4 * j, get_fr(&rd));
            if (rd.bad) {
                rc = PKO_WHIR_REJECT_FORMAT;
                goto done;
            }
            pko_transcript_absorb(t, ans + 4 * j);
        }
        if (p->pow_bits && (rc = pow_verify(t, &rd, p->pow_bits))) goto done;
        reverse_fr(ralpha, r_all + 4 * (nr - k), k);
        if ((rc = stir_verify(t, &rd, q, (size_t)1 << rows_log(p, r), k, r == 0 ? Bn : 1, bp,
                              prev_root, ralpha, folds, rc_r->pts + 4 * o)))
            goto done;
        pko_transcript_squeeze(t, gamma);
        powers(rc_r->coef, gamma, o + q);
        for (unsigned j = 0; j < o; j++) {
            pko_fr_mul(x, rc_r->coef + 4 * j, ans + 4 * j);
            pko_fr_add(last, last, x);
        }
        for (size_t i = 0; i < q; i++) {
            pko_fr_mul(x, rc_r->coef + 4 * (o + i), folds + 4 * i);
            pko_fr_add(last, last, x);
        }
        if ((rc = sc_verify(t, &rd, k, last, r_all + 4 * nr))) goto done;
        nr += k;
    }
    /* final polynomial */
    for (size_t i = 0; i < ((size_t)1 << nf); i++) {
        cp4(fc + 4 * i, get_fr(&rd));
        if (rd.bad) {
            rc = PKO_WHIR_REJECT_FORMAT;
            goto done;
        }
        pko_transcript_absorb(t, fc + 4 * i);
    }
    if (p->final_pow_bits && (rc = pow_verify(t, &rd, p->final_pow_bits))) goto done;
    {
        const size_t q = p->queries[R];
        reverse_fr(ralpha, r_all + 4 * (nr - k), k);
        if ((rc = stir_verify(t, &rd, q, (size_t)1 << rows_log(p, R), k, R == 0 ? Bn : 1, bp, root,
                              ralpha, folds, ypts)))
            goto done;
        for (size_t i = 0; i < q; i++) {
            pko_poly_eval(x, fc, (size_t)1 << nf, ypts + 4 * i);
            if (!eq4(x, folds + 4 * i)) {
                rc = PKO_WHIR_REJECT_FINAL_POLY;
                goto done;
            }
        }
    }
    if ((rc = sc_verify(t, &rd, nf, last, r_all + 4 * nr))) goto done;
    nr += nf;
    if (rd.bad || rd.pos != rd.len || nr != n) {
        rc = PKO_WHIR_REJECT_FORMAT;
        goto done;
    }
    {
        /* W(r): the initial OOD terms, the linear statements' weights (the
         * multilinear extension of mobius^T of their combination), each
         * round's OOD and STIR terms on the variables still live then. */
        uint64_t W[4] = {0, 0, 0, 0}, e[4];
        for (unsigned j = 0; j < o; j++) {
            eq_expand(e, z0 + 4 * j, r_all, n);
            pko_fr_mul(e, e, pw0 + 4 * j);
            pko_fr_add(W, W, e);
        }
        for (size_t a = 0; a < ncov; a++) {
            const uint64_t *av = covectors + 4 * N * a;
            for (size_t b = 0; b < N; b++) {
                pko_fr_mul(x, pw0 + 4 * (o + a), av + 4 * b);
                pko_fr_add(lin + 4 * b, lin + 4 * b, x);
            }
        }
        pko_subset_mobius_t(lin, n);
        size_t size = N;
        for (unsigned i = 0; i < n; i++) {
            const size_t h = size / 2;
            for (size_t b = 0; b < h; b++) {
                uint64_t d[4];
                pko_fr_sub(d, lin + 4 * (b + h), lin + 4 * b);
                pko_fr_mul(d, d, r_all + 4 * i);
                pko_fr_add(lin + 4 * b, lin + 4 * b, d);
            }
            size = h;
        }
        pko_fr_add(W, W, lin);
        for (unsigned r = 0; r < R; r++) {
            const round_claims *c = &rounds[r];
            for (size_t j = 0; j < c->npts; j++) {
                eq_expand(e, c->pts + 4 * j, r_all + 4 * (n - c->nv), c->nv);
                pko_fr_mul(e, e, c->coef + 4 * j);
                pko_fr_add(W, W, e);
            }
        }
        /* f(r) from the final coefficients: bind the top variable first */
        size = (size_t)1 << nf;
        for (unsigned i = 0; i < nf; i++) {
            const size_t h = size / 2;
            for (size_t b = 0; b < h; b++) {
                pko_fr_mul(x, fc + 4 * (b + h), r_all + 4 * (n - nf + i));
                pko_fr_add(fc + 4 * b, fc + 4 * b, x);
            }
            size = h;
        }
        pko_fr_mul(x, W, fc);
        if (!eq4(x, last)) rc = PKO_WHIR_REJECT_FINAL_CLAIM;
    }
done:
    for (unsigned r = 0; r < PKO_WHIR_MAX_ROUNDS; r++) {
        free(rounds[r].pts);
        free(rounds[r].coef);
    }
    free(r_all);
    free(pw0);
    free(z0);
    free(folds);
    free(ypts);
    free(fc);
    free(lin);
    return rc;
}
