/*
 * pk_oracle.c -- CPU restatement of ProveKit's Spartan+WHIR prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see pk_oracle.h).  Every function cites the
 * reference file:line it restates.  Arithmetic is exact modular integer
 * arithmetic over BN254 Fr, so any evaluation order gives identical bytes;
 * loops are parallelised with OpenMP where the reference uses rayon.
 */
#include "pk_oracle.h"
#include "poseidon2_t4_constants.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* BN254 Fr modulus, multiples and Montgomery constants
 * (skyscraper/core/src/constants.rs:8-15, bn254-multiplier/src/constants.rs). */
static const uint64_t P[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                              0xb85045b68181585dULL, 0x30644e72e131a029ULL};
static const uint64_t MODULUS[6][4] = {
    {0, 0, 0, 0},
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    {0x87c3eb27e0000002ULL, 0x5067d090f372e122ULL, 0x70a08b6d0302b0baULL, 0x60c89ce5c2634053ULL},
    {0xcba5e0bbd0000003ULL, 0x789bb8d96d2c51b3ULL, 0x28f0d12384840917ULL, 0x912ceb58a394e07dULL},
    {0x0f87d64fc0000004ULL, 0xa0cfa121e6e5c245ULL, 0xe14116da06056174ULL, 0xc19139cb84c680a6ULL},
    {0x5369cbe3b0000005ULL, 0xc903896a609f32d6ULL, 0x99915c908786b9d1ULL, 0xf1f5883e65f820d0ULL},
};
static const uint64_t INV64 = 0xc2e1f593efffffffULL; /* -p^-1 mod 2^64 */
static const uint64_t R2[4] = {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL,
                               0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL};
static const uint64_t ONE_MONT[4] = {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL,
                                     0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL};

/* Skyscraper round constants, canonical LE (skyscraper/core/src/constants.rs:30-49). */
static const uint64_t SKY_RC[18][4] = {
    {0, 0, 0, 0},
    {0x903c4324270bd744ULL, 0x873125f708a7d269ULL, 0x081dd27906c83855ULL, 0x276b1823ea6d7667ULL},
    {0x7ac8edbb4b378d71ULL, 0xe29d79f3d99e2cb7ULL, 0x751417914c1a5a18ULL, 0x0cf02bd758a484a6ULL},
    {0xfa7adc6769e5bc36ULL, 0x1c3f8e297cca387dULL, 0x0eb7730d63481db0ULL, 0x25b0e03f18ede544ULL},
    {0x57847e652f03cfb7ULL, 0x33440b9668873404ULL, 0x955a32e849af80bcULL, 0x002882fcbe14ae70ULL},
    {0x979231396257d4d7ULL, 0x29989c3e1b37d3c1ULL, 0x12ef02b47f1277baULL, 0x039ad8571e2b7a9cULL},
    {0xb5b48465abbb7887ULL, 0xa72a6bc5e6ba2d2bULL, 0x4cd48043712f7b29ULL, 0x1142d5410fc1fc1aULL},
    {0x7ab2c156059075d3ULL, 0x17cb3594047999b2ULL, 0x44f2c93598f289f7ULL, 0x1d78439f69bc0becULL},
    {0x05d7a965138b8edbULL, 0x36ef35a3d55c48b1ULL, 0x8ddfb8a1ac6f1628ULL, 0x258588a508f4ff82ULL},
    {0x1596fb9afccb49e9ULL, 0x9a7367d69a09a95bULL, 0x9bc43f6984e4c157ULL, 0x13087879d2f514feULL},
    {0x295ccd233b4109faULL, 0xe1d72f89ed868012ULL, 0x2e9e1eea4bc88a8eULL, 0x17dadee898c45232ULL},
    {0x9a8590b4aa1f486fULL, 0xb75834b430e9130eULL, 0xb8e90b1034d5de31ULL, 0x295c6d1546e7f4a6ULL},
    {0x850adcb74c6eb892ULL, 0x07699ef305b92fc3ULL, 0x4ef96a2ba1720f2dULL, 0x1288ca0e1d3ed446ULL},
    {0x01960f9349d1b5eeULL, 0x8ccad30769371c69ULL, 0xe5c81e8991c98662ULL, 0x17563b4d1ae023f3ULL},
    {0x6ba01e9476b32917ULL, 0xa1cb0a3add977bc9ULL, 0x86815a945815f030ULL, 0x2869043be91a1eeaULL},
    {0x81776c885511d976ULL, 0x7475d34f47f414e7ULL, 0x5d090056095d96cfULL, 0x14941f0aff59e79aULL},
    {0xbc40b4fd8fc8c034ULL, 0xbb7142c3cce4fd48ULL, 0x318356758a39005aULL, 0x1ce337a190f4379fULL},
    {0, 0, 0, 0},
};

/* ======================================================================= */
/* 256-bit helpers                                                          */
/* ======================================================================= */
static inline int geq(const uint64_t a[4], const uint64_t b[4]) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}
static inline int less_than(const uint64_t a[4], const uint64_t b[4]) { return !geq(a, b); }

static inline uint64_t add4(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
    u128 c = 0;
    for (int i = 0; i < 4; i++) { c += (u128)a[i] + b[i]; r[i] = (uint64_t)c; c >>= 64; }
    return (uint64_t)c;
}
static inline uint64_t sub4(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return borrow;
}
static inline void cpy4(uint64_t r[4], const uint64_t a[4]) { memcpy(r, a, 32); }

/* ======================================================================= */
/* Fr arithmetic (ark-ff semantics: Montgomery R = 2^256, fully reduced).   */
/* Multiplication is word-level CIOS (Koc, Acar, Kaliski 1996) with 64-bit  */
/* words; the result is reduced to [0, p) for any 256-bit inputs.           */
/* ======================================================================= */
void pko_fr_mul(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a[j] * b[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * INV64;
        c = (u128)m * P[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * P[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    /* t < 2^256 + p: subtract p until below it */
    while (t[4] != 0 || geq(t, P)) {
        uint64_t bw = sub4(t, t, P);
        t[4] -= bw;
    }
    cpy4(r, t);
}

void pko_fr_add(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
    uint64_t t[4];
    add4(t, a, b); /* a, b < p < 2^254: no carry out */
    if (geq(t, P)) sub4(t, t, P);
    cpy4(r, t);
}

void pko_fr_sub(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
    uint64_t t[4];
    if (sub4(t, a, b)) add4(t, t, P);
    cpy4(r, t);
}

void pko_fr_to_mont(uint64_t r[4], const uint64_t a[4]) { pko_fr_mul(r, a, R2); }

void pko_fr_from_mont(uint64_t r[4], const uint64_t a[4]) {
    static const uint64_t one[4] = {1, 0, 0, 0};
    pko_fr_mul(r, a, one);
}

static void fr_pow(uint64_t r[4], const uint64_t base[4], const uint64_t e[4]) {
    uint64_t acc[4], b[4];
    cpy4(acc, ONE_MONT);
    cpy4(b, base);
    for (int i = 0; i < 256; i++) {
        if ((e[i / 64] >> (i % 64)) & 1) pko_fr_mul(acc, acc, b);
        pko_fr_mul(b, b, b);
    }
    cpy4(r, acc);
}

static void fr_pow_u64(uint64_t r[4], const uint64_t base[4], uint64_t e) {
    uint64_t ee[4] = {e, 0, 0, 0};
    fr_pow(r, base, ee);
}

void pko_fr_inv(uint64_t r[4], const uint64_t a[4]) {
    uint64_t e[4];
    static const uint64_t two[4] = {2, 0, 0, 0};
    sub4(e, P, two);
    fr_pow(r, a, e);
}

static void fr_from_u64(uint64_t r[4], uint64_t v) {
    uint64_t c[4] = {v, 0, 0, 0};
    pko_fr_to_mont(r, c);
}

void pko_to_mont_many(uint64_t *v, size_t n) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) pko_fr_to_mont(v + 4 * i, v + 4 * i);
}
void pko_from_mont_many(uint64_t *v, size_t n) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) pko_fr_from_mont(v + 4 * i, v + 4 * i);
}

/* Fr::get_root_of_unity(n) for n = 2^k, k <= 28, as ark-ff derives it: the
 * two-adic root GENERATOR^((p-1)/2^28) with GENERATOR = 5 (ark-bn254 FrConfig),
 * squared 28-k times (used by ntt/src/ntt.rs:64, 287 and
 * provekit/common/src/ntt.rs:102-104). */
void pko_fr_root_of_unity(uint64_t r[4], uint64_t n) {
    int k = 0;
    while (((uint64_t)1 << k) < n) k++;
    uint64_t t[4], one[4] = {1, 0, 0, 0};
    sub4(t, P, one);
    for (int i = 0; i < 28; i++) { /* t = (p-1) >> 28 */
        t[0] = (t[0] >> 1) | (t[1] << 63);
        t[1] = (t[1] >> 1) | (t[2] << 63);
        t[2] = (t[2] >> 1) | (t[3] << 63);
        t[3] >>= 1;
    }
    uint64_t g[4];
    fr_from_u64(g, 5);
    fr_pow(r, g, t);
    for (int i = k; i < 28; i++) pko_fr_mul(r, r, r);
}

/* ======================================================================= */
/* ChaCha20 sampler                                                         */
/* ======================================================================= */
static inline uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
#define QR(a, b, c, d)                                   \
    do {                                                 \
        a += b; d ^= a; d = rotl32(d, 16);               \
        c += d; b ^= c; b = rotl32(b, 12);               \
        a += b; d ^= a; d = rotl32(d, 8);                \
        c += d; b ^= c; b = rotl32(b, 7);                \
    } while (0)

static void chacha20_block_n(const uint32_t key[8], uint64_t counter, uint32_t nonce,
                             uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)counter, (uint32_t)(counter >> 32), nonce, 0u};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    for (int i = 0; i < 10; i++) {
        QR(x[0], x[4], x[8], x[12]);
        QR(x[1], x[5], x[9], x[13]);
        QR(x[2], x[6], x[10], x[14]);
        QR(x[3], x[7], x[11], x[15]);
        QR(x[0], x[5], x[10], x[15]);
        QR(x[1], x[6], x[11], x[12]);
        QR(x[2], x[7], x[8], x[13]);
        QR(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

static void chacha20_block(const uint32_t key[8], uint64_t counter, uint32_t out[16]) {
    chacha20_block_n(key, counter, 0u, out);
}

void pko_sample_fr_indexed(uint64_t seed, uint64_t start, size_t n, uint64_t *out) {
    const uint32_t key[8] = {(uint32_t)seed, (uint32_t)(seed >> 32), 0, 0, 0, 0, 0, 0};
    const uint64_t two253[4] = {0, 0, 0, (uint64_t)1 << 61};
    uint64_t t[4];
    pko_fr_to_mont(t, two253);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
        uint32_t blk[16];
        uint64_t lo[4], hi[4], a[4], b[4];
        chacha20_block_n(key, start + i, 1u, blk);
        for (int j = 0; j < 4; j++) {
            lo[j] = (uint64_t)blk[2 * j] | ((uint64_t)blk[2 * j + 1] << 32);
            hi[j] = (uint64_t)blk[8 + 2 * j] | ((uint64_t)blk[8 + 2 * j + 1] << 32);
        }
        lo[3] &= ((uint64_t)1 << 61) - 1;
        hi[3] &= ((uint64_t)1 << 61) - 1;
        pko_fr_to_mont(a, lo);
        pko_fr_to_mont(b, hi);
        pko_fr_mul(b, b, t);
        pko_fr_add(out + 4 * i, a, b);
    }
}

void pko_sample_fr(uint64_t seed, size_t n, uint64_t *out, int mont) {
    uint32_t key[8] = {(uint32_t)seed, (uint32_t)(seed >> 32), 0, 0, 0, 0, 0, 0};
    uint64_t counter = 0;
    size_t got = 0;
    uint32_t blk[16];
    while (got < n) {
        chacha20_block(key, counter++, blk);
        for (int h = 0; h < 2 && got < n; h++) {
            uint64_t v[4];
            for (int i = 0; i < 4; i++)
                v[i] = (uint64_t)blk[8 * h + 2 * i] | ((uint64_t)blk[8 * h + 2 * i + 1] << 32);
            v[3] &= 0x3fffffffffffffffULL;
            if (geq(v, P)) continue;
            if (mont) pko_fr_to_mont(out + 4 * got, v);
            else cpy4(out + 4 * got, v);
            got++;
        }
    }
}

/* ======================================================================= */
/* ntt crate                                                                */
/* ======================================================================= */
static size_t reverse_bits(size_t v, int bits) {
    size_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((v >> i) & 1) << (bits - 1 - i);
    return r;
}
static int log2_exact(size_t n) {
    int k = 0;
    while (((size_t)1 << k) < n) k++;
    return k;
}
static int is_pow2(size_t n) { return n && !(n & (n - 1)); }

/* init_roots_reverse_ordered (ntt/src/ntt.rs:275-306): roots[bitrev(i)] = w^i
 * for i < order/2.  A table of larger order has this one as prefix. */
void pko_roots_reverse_ordered(uint64_t *out, size_t order) {
    size_t n = order / 2;
    if (n == 0) return;
    if (n == 1) { cpy4(out, ONE_MONT); return; }
    uint64_t w[4];
    pko_fr_root_of_unity(w, order);
    int bits = log2_exact(n);
    /* parallel: w^i computed per chunk */
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    size_t chunk = (n + nt - 1) / nt;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nt; t++) {
        size_t lo = (size_t)t * chunk, hi = lo + chunk < n ? lo + chunk : n;
        if (lo >= hi) continue;
        uint64_t wk[4];
        fr_pow_u64(wk, w, lo);
        for (size_t i = lo; i < hi; i++) {
            cpy4(out + 4 * reverse_bits(i, bits), wk);
            pko_fr_mul(wk, wk, w);
        }
    }
}

static inline void butterfly(uint64_t *e, uint64_t *o, const uint64_t w[4]) {
    uint64_t t[4];
    pko_fr_mul(t, w, o);
    uint64_t ev[4];
    cpy4(ev, e);
    pko_fr_add(e, ev, t);
    pko_fr_sub(o, ev, t);
}

/* ntt_nr / interleaved_ntt_nr / dit_nr_cache (ntt/src/ntt.rs:105-108,
 * 150-248): radix-2 DIT, normal order in, bit-reversed order out; the stage
 * with G groups pairs element i of group k with i + half and uses twiddle
 * roots[k]; the first log2(num_groups) stages are skipped.
 * Returns 0, or -1 where the reference panics (plus two documented
 * rejections: len not a multiple of codeword_size, non-power-of-two
 * num_groups). */
int pko_ntt_nr(uint64_t *values, size_t len, size_t codeword_size, size_t num_groups) {
    if (codeword_size <= 1) return 0;
    if (num_groups == 0 || len % num_groups) return -1;
    if (!is_pow2(codeword_size) || !is_pow2(num_groups)) return -1;
    if (len == 0 || len % codeword_size) return -1;
    if (num_groups >= codeword_size) return 0;
    size_t half_order = codeword_size / 2;
    uint64_t *roots = (uint64_t *)malloc(32 * half_order);
    if (!roots) return -2;
    pko_roots_reverse_ordered(roots, codeword_size);
    /* Phases A/B (ntt.rs:189-219): whole-array stages while a group is
     * larger than the 32 KiB workload; phase C (ntt.rs:221-248): every
     * group finishes its remaining stages locally (dit_nr_cache). */
    const size_t workload = 1024; /* workload_size::<Fr>() */
    size_t eig = len / num_groups;
    size_t groups = num_groups;
    for (; groups < codeword_size && eig > workload; groups *= 2, eig /= 2) {
        size_t half = eig / 2;
        size_t total = groups * half;
#pragma omp parallel for schedule(static)
        for (size_t x = 0; x < total; x++) {
            size_t k = x / half, i = x % half;
            uint64_t *e = values + 4 * (k * eig + i);
            butterfly(e, e + 4 * half, roots + 4 * k);
        }
    }
    size_t size = codeword_size / groups;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t seg = 0; seg < groups; seg++) {
        uint64_t *in = values + 4 * seg * eig;
        size_t e2 = eig;
        for (size_t ng = 1; ng < size; ng *= 2, e2 /= 2) {
            size_t half = e2 / 2;
            for (size_t k = 0; k < ng; k++) {
                const uint64_t *w = roots + 4 * (seg * ng + k);
                for (size_t i = 0; i < half; i++)
                    butterfly(in + 4 * (k * e2 + i), in + 4 * (k * e2 + half + i), w);
            }
        }
    }
    free(roots);
    return 0;
}

static void reverse_order(uint64_t *v, size_t n) {
    if (n <= 1) return;
    int bits = log2_exact(n);
    for (size_t i = 0; i < n; i++) {
        size_t r = reverse_bits(i, bits);
        if (i < r) {
            uint64_t t[4];
            cpy4(t, v + 4 * i);
            cpy4(v + 4 * i, v + 4 * r);
            cpy4(v + 4 * r, t);
        }
    }
}

/* intt_rn / intt_nr (ntt/src/ntt.rs:326-348). */
int pko_intt_rn(uint64_t *values, size_t len) {
    if (!is_pow2(len)) return -1; /* reverse_order asserts a power of two */
    reverse_order(values, len);
    /* values[1..].reverse() */
    for (size_t i = 1, j = len - 1; i < j; i++, j--) {
        uint64_t t[4];
        cpy4(t, values + 4 * i);
        cpy4(values + 4 * i, values + 4 * j);
        cpy4(values + 4 * j, t);
    }
    int rc = pko_ntt_nr(values, len, len, 1);
    if (rc) return rc;
    uint64_t f[4];
    fr_from_u64(f, len);
    pko_fr_inv(f, f);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < len; i++) pko_fr_mul(values + 4 * i, values + 4 * i, f);
    reverse_order(values, len);
    return 0;
}

/* ======================================================================= */
/* RSFr (provekit/common/src/ntt.rs)                                        */
/* ======================================================================= */
static size_t next_pow2(size_t v) {
    size_t r = 1;
    while (r < v) r <<= 1;
    return r;
}

int pko_rs_interleaved_encode(const uint64_t *messages, size_t num_messages,
                              size_t message_length, const uint64_t *masks,
                              size_t mask_len, size_t codeword_length, uint64_t *out) {
    if (num_messages == 0) return 0;                                   /* :57-59 */
    size_t total = num_messages * codeword_length;                     /* :68 */
    if (message_length > codeword_length) return -1;
    if (message_length * num_messages + mask_len > total) return -1;   /* :79-80 */
    memset(out, 0, 32 * total);
#pragma omp parallel for schedule(static)
    for (size_t col = 0; col < message_length; col++)                  /* :72-77 */
        for (size_t row = 0; row < num_messages; row++)
            cpy4(out + 4 * (col * num_messages + row), messages + 4 * (row * message_length + col));
    if (mask_len) memcpy(out + 4 * message_length * num_messages, masks, 32 * mask_len);
    size_t mask_length = mask_len / num_messages;                      /* :82 */
    size_t coset_size = next_pow2(message_length + mask_length);       /* :86 */
    if (coset_size > ((size_t)1 << 28)) return -1;
    while (codeword_length % coset_size) {                             /* :87-89 */
        coset_size = next_pow2(coset_size + 1);
        if (coset_size > ((size_t)1 << 28)) return -1;
    }
    size_t num_cosets = codeword_length / coset_size;
    size_t chunk = coset_size * num_messages;                          /* :92-95 */
    for (size_t k = 1; k < num_cosets; k++) memcpy(out + 4 * k * chunk, out, 32 * chunk);
    if (codeword_length <= 1) return 0;
    return pko_ntt_nr(out, total, codeword_length, num_cosets);        /* :97 */
}

/* evaluation_points (provekit/common/src/ntt.rs:22-42). */
void pko_rs_evaluation_points(size_t codeword_length, const size_t *indices, size_t n,
                              uint64_t *out) {
    int bits = 0;
    while (bits < 64 && (((size_t)1 << bits) < codeword_length)) bits++;
    uint64_t g[4];
    pko_fr_root_of_unity(g, codeword_length);
    for (size_t x = 0; x < n; x++) {
        size_t k = bits == 0 ? indices[x] : reverse_bits(indices[x] & (((size_t)1 << bits) - 1), bits);
        fr_pow_u64(out + 4 * x, g, k);
    }
}

/* ======================================================================= */
/* Skyscraper v2                                                            */
/* ======================================================================= */
/* reduce_partial (skyscraper/core/src/reduce.rs:34-41) */
static inline void reduce_partial(uint64_t x[4]) {
    uint64_t mult = x[3] / (MODULUS[1][3] + 1);
    sub4(x, x, MODULUS[mult]);
}
/* reduce_1 (reduce.rs:23-31) */
static inline void reduce_1(uint64_t x[4]) {
    uint64_t r[4];
    if (!sub4(r, x, MODULUS[1])) cpy4(x, r);
}
static inline void reduce_full(uint64_t x[4]) { reduce_partial(x); reduce_1(x); }

/* reduce_partial_add_rc (reduce.rs:48-55): x - (k*p - rc) with k from the
 * top limb (wrapping for k = 0, i.e. x + rc). */
static inline void reduce_partial_add_rc(uint64_t x[4], int rc) {
    uint64_t mult = x[3] / (MODULUS[1][3] + 1);
    uint64_t m[4];
    sub4(m, MODULUS[mult], SKY_RC[rc]);
    sub4(x, x, m);
}

uint8_t pko_sky_sbox(uint8_t v) { /* skyscraper/core/src/bar.rs:40-42 */
    uint8_t nv = (uint8_t)~v;
    uint8_t r1 = (uint8_t)((nv << 1) | (nv >> 7));
    uint8_t r2 = (uint8_t)((v << 2) | (v >> 6));
    uint8_t r3 = (uint8_t)((v << 3) | (v >> 5));
    uint8_t t = (uint8_t)(v ^ (r1 & r2 & r3));
    return (uint8_t)((t << 1) | (t >> 7));
}

/* bar (skyscraper/core/src/bar.rs:15-31): input < 2p. */
static void bar(uint64_t x[4]) {
    reduce_1(x);
    uint64_t y[4] = {x[2], x[3], x[0], x[1]};
    uint8_t *b = (uint8_t *)y;
    for (int i = 0; i < 32; i++) b[i] = pko_sky_sbox(b[i]);
    reduce_partial(y);
    cpy4(x, y);
}

/* Montgomery square x^2 * 2^-256 mod p, the value bn254_multiplier::scalar_sqr
 * (bn254-multiplier/src/scalar.rs:12-70) computes; every later step of the
 * compression depends only on its value mod p. */
static inline void msq(uint64_t r[4], const uint64_t x[4]) { pko_fr_mul(r, x, x); }

/* generic::compress (skyscraper/core/src/generic.rs:77-102). */
void pko_sky_compress(uint64_t out[4], const uint64_t lin[4], const uint64_t rin[4]) {
    static const int is_bar[18] = {0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 0, 0, 0, 0};
    uint64_t l[4], r[4], t[4], f[4], nl[4];
    cpy4(l, lin); reduce_partial(l);
    cpy4(r, rin); reduce_partial(r);
    cpy4(t, l);
    /* round 0 */
    msq(f, l);
    add4(nl, r, f);
    reduce_partial(nl);
    cpy4(r, l); cpy4(l, nl);
    for (int k = 1; k < 17; k++) {
        if (is_bar[k]) { cpy4(f, l); bar(f); }
        else msq(f, l);
        add4(nl, r, f);
        reduce_partial_add_rc(nl, k);
        cpy4(r, l); cpy4(l, nl);
    }
    msq(f, l);
    add4(nl, r, f);
    add4(nl, nl, t);
    reduce_full(nl);
    cpy4(out, nl);
}

/* simple::compress_many via generic::compress_many (generic.rs:14-37). */
int pko_sky_compress_many(const uint8_t *messages, size_t n, uint8_t *hashes) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
        uint64_t l[4], r[4], o[4];
        memcpy(l, messages + 64 * i, 32);
        memcpy(r, messages + 64 * i + 32, 32);
        pko_sky_compress(o, l, r);
        memcpy(hashes + 32 * i, o, 32);
    }
    return 0;
}

/* Canonical-domain field helpers for reference::permute, whose ark code
 * computes l.square() * SIGMA_INV with SIGMA_INV = 2^-256 mod p; on canonical
 * values that is exactly the Montgomery square. */
static void canon_add3(uint64_t r[4], const uint64_t a[4], const uint64_t b[4], const uint64_t c[4]) {
    uint64_t t[4];
    pko_fr_add(t, a, b);
    pko_fr_add(r, t, c);
}

static void ref_bar(uint64_t out[4], const uint64_t x[4]) { /* reference.rs:80-94 */
    uint64_t y[4] = {x[2], x[3], x[0], x[1]};
    uint8_t *b = (uint8_t *)y;
    for (int i = 0; i < 32; i++) b[i] = pko_sky_sbox(b[i]);
    reduce_full(y); /* from_le_bytes_mod_order */
    cpy4(out, y);
}

void pko_sky_ss(int round, uint64_t l[4], uint64_t r[4]) { /* reference.rs:63-69 */
    uint64_t f[4], t[4];
    for (int h = 0; h < 2; h++) {
        msq(f, l);
        canon_add3(r, r, f, SKY_RC[round + h]);
        cpy4(t, l); cpy4(l, r); cpy4(r, t);
    }
}

void pko_sky_bb(int round, uint64_t l[4], uint64_t r[4]) { /* reference.rs:72-78 */
    uint64_t f[4], t[4];
    for (int h = 0; h < 2; h++) {
        ref_bar(f, l);
        canon_add3(r, r, f, SKY_RC[round + h]);
        cpy4(t, l); cpy4(l, r); cpy4(r, t);
    }
}

void pko_sky_permute(uint64_t l[4], uint64_t r[4]) { /* reference.rs:49-60 */
    pko_sky_ss(0, l, r);
    pko_sky_ss(2, l, r);
    pko_sky_ss(4, l, r);
    pko_sky_bb(6, l, r);
    pko_sky_ss(8, l, r);
    pko_sky_bb(10, l, r);
    pko_sky_ss(12, l, r);
    pko_sky_ss(14, l, r);
    pko_sky_ss(16, l, r);
}

/* SkyscraperHashEngine::hash_many (provekit/common/src/skyscraper/whir.rs:42-100):
 * size 32 copies, size 64 compresses, larger sizes left-fold 32-byte chunks. */
int pko_hash_many(size_t size, const uint8_t *input, size_t count, uint8_t *output) {
    if (size == 0 || size % 32) return -1;
    if (size == 32) { memcpy(output, input, 32 * count); return 0; }
    if (size == 64) return pko_sky_compress_many(input, count, output);
    size_t chunks = size / 32;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < count; i++) {
        const uint8_t *msg = input + i * size;
        uint64_t acc[4], e[4];
        memcpy(acc, msg, 32);
        memcpy(e, msg + 32, 32);
        pko_sky_compress(acc, acc, e);
        for (size_t k = 2; k < chunks; k++) {
            memcpy(e, msg + 32 * k, 32);
            pko_sky_compress(acc, acc, e);
        }
        memcpy(output + 32 * i, acc, 32);
    }
    return 0;
}

/* Binary Merkle tree: leaf digests via hash_many(leaf_size), internal nodes
 * via hash_many(64) of (left || right) -- the engine calls WHIR's tree makes
 * (skyscraper/whir.rs:62-70), and the layout the Go verifier recomputes
 * (recursive-verifier/app/circuit/whir_utilities.go:14-47). */
int pko_merkle_tree(const uint8_t *leaves, size_t leaf_size, size_t count, uint8_t *layers) {
    if (!is_pow2(count)) return -1;
    int rc = pko_hash_many(leaf_size, leaves, count, layers);
    if (rc) return rc;
    uint8_t *cur = layers;
    size_t n = count;
    while (n > 1) {
        uint8_t *next = cur + 32 * n;
        pko_sky_compress_many(cur, n / 2, next);
        cur = next;
        n /= 2;
    }
    return 0;
}

/* generic::solve (skyscraper/core/src/generic.rs:42-71): smallest nonce whose
 * compress([challenge, [nonce,0,0,0]]) is below threshold. */
uint64_t pko_sky_pow_solve(const uint64_t challenge[4], const uint64_t threshold[4]) {
    for (uint64_t nonce = 0;; nonce++) {
        uint64_t r[4] = {nonce, 0, 0, 0}, h[4];
        pko_sky_compress(h, challenge, r);
        if (less_than(h, threshold)) return nonce;
    }
}

/* ======================================================================= */
/* Spartan sumcheck helpers (provekit/common/src/utils/sumcheck.rs)         */
/* ======================================================================= */
/* calculate_eq (sumcheck.rs:182-188) */
void pko_calculate_eq(uint64_t out[4], const uint64_t *r, const uint64_t *alpha, size_t n) {
    uint64_t acc[4], t1[4], t2[4], omr[4], oma[4];
    cpy4(acc, ONE_MONT);
    for (size_t i = 0; i < n; i++) {
        pko_fr_mul(t1, r + 4 * i, alpha + 4 * i);
        pko_fr_sub(omr, ONE_MONT, r + 4 * i);
        pko_fr_sub(oma, ONE_MONT, alpha + 4 * i);
        pko_fr_mul(t2, omr, oma);
        pko_fr_add(t1, t1, t2);
        pko_fr_mul(acc, acc, t1);
    }
    cpy4(out, acc);
}

/* calculate_evaluations_over_boolean_hypercube_for_eq / eval_eq
 * (sumcheck.rs:108-153): out[x] = prod_i (bit_i(x) ? r_i : 1 - r_i), with
 * r_0 bound to the most significant bit, truncated to num_entries. */
int pko_eq_hypercube(const uint64_t *r, size_t nr, size_t num_entries, uint64_t *out) {
    if (num_entries == 0) return 0;
    if (nr >= 64 || num_entries > ((size_t)1 << nr)) return -1;
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < num_entries; x++) {
        uint64_t acc[4], t[4];
        cpy4(acc, ONE_MONT);
        for (size_t i = 0; i < nr; i++) {
            int bit = (int)((x >> (nr - 1 - i)) & 1);
            if (bit) pko_fr_mul(acc, acc, r + 4 * i);
            else { pko_fr_sub(t, ONE_MONT, r + 4 * i); pko_fr_mul(acc, acc, t); }
        }
        cpy4(out + 4 * x, acc);
    }
    return 0;
}

/* One round of run_zk_sumcheck_prover's map-reduce
 * (provekit/prover/src/whir_r1cs.rs:551-559) over sumcheck_fold_map_reduce
 * (sumcheck.rs:14-102).  Without fold: pairs (t[i], t[i+size/2]).  With fold:
 * quarter layout, t[i] += f*(t[i+2q]-t[i]), t[i+q] += f*(t[i+3q]-t[i+q]),
 * pairs (t[i], t[i+q]); the live tables are then the first size/2 entries.
 * out = (f(0), f(-1), f(inf)) as 3 x 4 limbs. */
int pko_spartan_round(uint64_t *a, uint64_t *b, uint64_t *c, uint64_t *eq, size_t size,
                      const uint64_t *fold, uint64_t out[12]) {
    if (!is_pow2(size) || size < 2) return -1;
    if (fold && size < 4) return -1;
    uint64_t *tabs[4] = {a, b, c, eq};
    size_t npairs = fold ? size / 4 : size / 2;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    uint64_t *part = (uint64_t *)calloc((size_t)nt * 12, 8);
    if (!part) return -2;
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        uint64_t acc[12] = {0};
#pragma omp for schedule(static)
        for (size_t i = 0; i < npairs; i++) {
            uint64_t v0[4][4], v1[4][4];
            for (int j = 0; j < 4; j++) {
                uint64_t *t = tabs[j];
                if (fold) {
                    size_t q = size / 4;
                    uint64_t d[4];
                    pko_fr_sub(d, t + 4 * (i + 2 * q), t + 4 * i);
                    pko_fr_mul(d, fold, d);
                    pko_fr_add(t + 4 * i, t + 4 * i, d);
                    pko_fr_sub(d, t + 4 * (i + 3 * q), t + 4 * (i + q));
                    pko_fr_mul(d, fold, d);
                    pko_fr_add(t + 4 * (i + q), t + 4 * (i + q), d);
                    cpy4(v0[j], t + 4 * i);
                    cpy4(v1[j], t + 4 * (i + q));
                } else {
                    cpy4(v0[j], t + 4 * i);
                    cpy4(v1[j], t + 4 * (i + size / 2));
                }
            }
            /* closure at whir_r1cs.rs:552-558; order a, b, c, eq */
            uint64_t ab[4], f0[4], tmp[4], x[4], y[4], z[4], e2[4];
            pko_fr_mul(ab, v0[0], v0[1]);
            pko_fr_sub(ab, ab, v0[2]);
            pko_fr_mul(f0, v0[3], ab);
            /* (2*eq0 - eq1) * ((2a0-a1)(2b0-b1) - (2c0-c1)) */
            pko_fr_add(x, v0[0], v0[0]); pko_fr_sub(x, x, v1[0]);
            pko_fr_add(y, v0[1], v0[1]); pko_fr_sub(y, y, v1[1]);
            pko_fr_add(z, v0[2], v0[2]); pko_fr_sub(z, z, v1[2]);
            pko_fr_mul(tmp, x, y);
            pko_fr_sub(tmp, tmp, z);
            pko_fr_add(e2, v0[3], v0[3]); pko_fr_sub(e2, e2, v1[3]);
            uint64_t fm1[4];
            pko_fr_mul(fm1, e2, tmp);
            /* (eq1 - eq0)(a1 - a0)(b1 - b0) */
            uint64_t finf[4];
            pko_fr_sub(x, v1[3], v0[3]);
            pko_fr_sub(y, v1[0], v0[0]);
            pko_fr_sub(z, v1[1], v0[1]);
            pko_fr_mul(finf, x, y);
            pko_fr_mul(finf, finf, z);
            pko_fr_add(acc, acc, f0);
            pko_fr_add(acc + 4, acc + 4, fm1);
            pko_fr_add(acc + 8, acc + 8, finf);
        }
        memcpy(part + 12 * tid, acc, sizeof acc);
    }
    uint64_t res[12] = {0};
    for (int t = 0; t < nt; t++)
        for (int k = 0; k < 3; k++) pko_fr_add(res + 4 * k, res + 4 * k, part + 12 * t + 4 * k);
    memcpy(out, res, sizeof res);
    free(part);
    return 0;
}

/* HydratedSparseMatrix x &[Fr] (provekit/common/src/sparse_matrix.rs:606-627). */
int pko_spmv(const uint64_t *row_ptr, const uint32_t *cols, const uint64_t *vals, size_t num_rows,
             const uint64_t *x, uint64_t *y) {
#pragma omp parallel for schedule(static)
    for (size_t row = 0; row < num_rows; row++) {
        uint64_t acc[4] = {0, 0, 0, 0}, t[4];
        for (uint64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) {
            pko_fr_mul(t, vals + 4 * k, x + 4 * (size_t)cols[k]);
            pko_fr_add(acc, acc, t);
        }
        cpy4(y + 4 * row, acc);
    }
    return 0;
}

/* eval_cubic_poly (sumcheck.rs:156-158) */
void pko_eval_cubic(uint64_t out[4], const uint64_t poly[16], const uint64_t x[4]) {
    uint64_t acc[4];
    pko_fr_mul(acc, x, poly + 12);
    pko_fr_add(acc, acc, poly + 8);
    pko_fr_mul(acc, acc, x);
    pko_fr_add(acc, acc, poly + 4);
    pko_fr_mul(acc, acc, x);
    pko_fr_add(out, acc, poly);
}

/* compute_blinding_coefficients_for_round (provekit/prover/src/whir_r1cs.rs:427-492). */
void pko_blinding_coeffs(const uint64_t *g, size_t n, size_t compute_for, const uint64_t *alphas,
                         uint64_t out[16]) {
    int all_fixed = 0;
    size_t cf = compute_for;
    if (cf == n) { all_fixed = 1; cf = n - 1; }
    uint64_t prefix[4] = {0, 0, 0, 0}, suffix[4] = {0, 0, 0, 0}, t[4];
    for (size_t i = 0; i < cf; i++) {
        pko_eval_cubic(t, g + 16 * i, alphas + 4 * i);
        pko_fr_add(prefix, prefix, t);
    }
    static const uint64_t zero[4] = {0, 0, 0, 0};
    for (size_t i = cf + 1; i < n; i++) {
        uint64_t t0[4], t1[4];
        pko_eval_cubic(t0, g + 16 * i, zero);
        pko_eval_cubic(t1, g + 16 * i, ONE_MONT);
        pko_fr_add(suffix, suffix, t0);
        pko_fr_add(suffix, suffix, t1);
    }
    uint64_t pm[4], sm[4], two[4], inv2[4];
    cpy4(pm, ONE_MONT);
    for (size_t i = 0; i < n - 1 - cf; i++) pko_fr_add(pm, pm, pm);
    pko_fr_add(two, ONE_MONT, ONE_MONT);
    pko_fr_inv(inv2, two);
    pko_fr_mul(sm, pm, inv2);
    uint64_t cst[4];
    pko_fr_mul(cst, pm, prefix);
    pko_fr_mul(t, sm, suffix);
    pko_fr_add(cst, cst, t);
    const uint64_t *cur = g + 16 * cf;
    uint64_t res[16];
    pko_fr_mul(res, pm, cur);
    pko_fr_add(res, res, cst);
    for (int k = 1; k < 4; k++) pko_fr_mul(res + 4 * k, pm, cur + 4 * k);
    if (all_fixed) {
        uint64_t v[4];
        pko_eval_cubic(v, res, alphas + 4 * cf);
        memset(out, 0, 128);
        cpy4(out, v);
        return;
    }
    memcpy(out, res, 128);
}

/* whir::algebra::dot as used at whir_r1cs.rs:614-617, 637, 650. */
void pko_dot(uint64_t out[4], const uint64_t *a, const uint64_t *b, size_t n) {
    uint64_t acc[4] = {0, 0, 0, 0}, t[4];
    for (size_t i = 0; i < n; i++) {
        pko_fr_mul(t, a + 4 * i, b + 4 * i);
        pko_fr_add(acc, acc, t);
    }
    cpy4(out, acc);
}

int pko_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ======================================================================= */
/* Transcript stand-in and the Spartan zk-sumcheck driver                  */
/* ======================================================================= */
void pko_transcript_init(pko_transcript *t, const uint64_t domain[4]) {
    cpy4(t->l, domain);
    reduce_full(t->l);
    memset(t->r, 0, 32);
    pko_sky_permute(t->l, t->r);
}

void pko_transcript_absorb(pko_transcript *t, const uint64_t x_mont[4]) {
    uint64_t v[4];
    pko_fr_from_mont(v, x_mont);
    pko_fr_add(t->l, t->l, v);
    pko_sky_permute(t->l, t->r);
}

void pko_transcript_squeeze(pko_transcript *t, uint64_t out_mont[4]) {
    pko_sky_permute(t->l, t->r);
    pko_fr_to_mont(out_mont, t->l);
}

int pko_spartan_sumcheck(pko_transcript *t, uint64_t *a, uint64_t *b, uint64_t *c, size_t m0,
                         const uint64_t *g, const uint64_t *w1, size_t blinding_offset,
                         uint64_t *r_out, uint64_t rho_out[4], uint64_t sum_g_out[4],
                         uint64_t *coeffs_out, uint64_t *alpha_out, uint64_t blinding_eval[4]) {
    if (m0 < 1 || m0 > 30) return -1;
    size_t n = (size_t)1 << m0;
    for (size_t i = 0; i < m0; i++) pko_transcript_squeeze(t, r_out + 4 * i);   /* :529 */
    uint64_t *eq = (uint64_t *)malloc(32 * n);
    if (!eq) return -2;
    pko_eq_hypercube(r_out, m0, n, eq);                                        /* :530 */
    /* sum_over_hypercube (whir_r1cs.rs:494-501) */
    uint64_t g0[16], t0[4], t1[4], sum_g[4];
    static const uint64_t zero[4] = {0, 0, 0, 0};
    pko_blinding_coeffs(g, m0, 0, NULL, g0);
    pko_eval_cubic(t0, g0, zero);
    pko_eval_cubic(t1, g0, ONE_MONT);
    pko_fr_add(sum_g, t0, t1);
    cpy4(sum_g_out, sum_g);
    pko_transcript_absorb(t, sum_g);                                           /* :541 */
    uint64_t rho[4];
    pko_transcript_squeeze(t, rho);                                            /* :543 */
    cpy4(rho_out, rho);
    uint64_t saved[4];
    pko_fr_mul(saved, rho, sum_g);                                             /* :546 */
    uint64_t half[4], two[4];
    pko_fr_add(two, ONE_MONT, ONE_MONT);
    pko_fr_inv(half, two);
    size_t size = n;
    for (size_t idx = 0; idx < m0; idx++) {                                    /* :550-610 */
        uint64_t h[12];
        int rc = pko_spartan_round(a, b, c, eq, size, idx ? alpha_out + 4 * (idx - 1) : NULL, h);
        if (rc) { free(eq); return rc; }
        if (idx) size /= 2;
        uint64_t gp[16];
        pko_blinding_coeffs(g, m0, idx, alpha_out, gp);
        uint64_t cf[16], tmp[4], gem1[4], cem1[4];
        pko_fr_mul(tmp, rho, gp);
        pko_fr_add(cf, h, tmp);                                   /* c0 */
        pko_fr_sub(gem1, gp, gp + 4);
        pko_fr_add(gem1, gem1, gp + 8);
        pko_fr_sub(gem1, gem1, gp + 12);
        pko_fr_mul(tmp, rho, gem1);
        pko_fr_add(cem1, h + 4, tmp);
        pko_fr_add(tmp, saved, cem1);
        pko_fr_sub(tmp, tmp, cf);
        pko_fr_sub(tmp, tmp, cf);
        pko_fr_sub(tmp, tmp, cf);
        pko_fr_mul(cf + 8, half, tmp);                            /* c2 */
        pko_fr_mul(tmp, rho, gp + 12);
        pko_fr_add(cf + 12, h + 8, tmp);                          /* c3 */
        pko_fr_sub(tmp, saved, cf);
        pko_fr_sub(tmp, tmp, cf);
        pko_fr_sub(tmp, tmp, cf + 12);
        pko_fr_sub(cf + 4, tmp, cf + 8);                          /* c1 */
        memcpy(coeffs_out + 16 * idx, cf, 128);
        for (int k = 0; k < 4; k++) pko_transcript_absorb(t, cf + 4 * k);
        pko_transcript_squeeze(t, alpha_out + 4 * idx);
        pko_eval_cubic(saved, cf, alpha_out + 4 * idx);
    }
    free(eq);
    /* blinding_eval = <expand_powers::<4>(alpha), w1[offset..]> (:613-618) */
    uint64_t acc[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < m0; i++) {
        uint64_t pw[4], tt[4];
        cpy4(pw, ONE_MONT);
        for (int k = 0; k < 4; k++) {
            pko_fr_mul(tt, pw, w1 + 4 * (blinding_offset + 4 * i + k));
            pko_fr_add(acc, acc, tt);
            pko_fr_mul(pw, pw, alpha_out + 4 * i);
        }
    }
    cpy4(blinding_eval, acc);
    pko_transcript_absorb(t, acc);
    return 0;
}

/* ======================================================================= */
/* Spartan prove core                                                      */
/* ======================================================================= */
static size_t ceil_log2(size_t n) { /* utils::next_power_of_two (utils/mod.rs:71-79) */
    size_t p = 1, k = 0;
    while (p < n) { p <<= 1; k++; }
    return k;
}

void pko_r1cs_sizing(size_t num_constraints, size_t num_witnesses, size_t *m_out, size_t *m0_out) {
    size_t m = ceil_log2(num_witnesses), m0 = ceil_log2(num_constraints);
    if (m < 13) m = 13;                                   /* MIN_WHIR_NUM_VARIABLES */
    if (m0 < 1) m0 = 1;                                   /* MIN_SUMCHECK_NUM_VARIABLES */
    if (((size_t)1 << m) - num_witnesses < 4 * m0) m++;
    *m_out = m;
    *m0_out = m0;
}

/* splitmix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014): the integer choices of the synthetic R1CS. */
static uint64_t splitmix64_next(uint64_t *s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static uint64_t splitmix64_below(uint64_t *s, uint64_t n) {
    return n ? splitmix64_next(s) % n : 0;
}

int pko_synthetic_r1cs(uint64_t seed, size_t nc, size_t ni, uint64_t *row_ptr[3],
                       uint32_t *cols[3], uint64_t *vals[3], size_t nnz_out[3],
                       uint64_t *witness) {
    if (ni + nc + 1 >= ((size_t)1 << 32)) return -1;
    uint64_t rng = seed;
    /* the row structure first: every row's two nonzero counts */
    uint8_t *ka = malloc(nc ? nc : 1), *kb = malloc(nc ? nc : 1);
    size_t total = 0;
    for (size_t i = 0; i < nc; i++) {
        ka[i] = (uint8_t)(1 + splitmix64_below(&rng, 3));
        kb[i] = (uint8_t)(1 + splitmix64_below(&rng, 3));
        total += (size_t)ka[i] + kb[i];
    }
    uint64_t *coef = malloc(32 * (total ? total : 1));
    pko_sample_fr(seed + 1, total, coef, 1);
    cpy4(witness, ONE_MONT);
    pko_sample_fr(seed, ni, witness + 4, 1);
    size_t e[2] = {0, 0}, used = 0;
    row_ptr[0][0] = row_ptr[1][0] = row_ptr[2][0] = 0;
    for (size_t i = 0; i < nc; i++) {
        const uint64_t hi = ni + i + 1; /* columns in [0, ni + i] */
        uint64_t dot[2][4];
        for (int m = 0; m < 2; m++) {
            const int k = m == 0 ? ka[i] : kb[i];
            uint64_t acc[4] = {0, 0, 0, 0}, t[4];
            for (int j = 0; j < k; j++) {
                const uint32_t col = (uint32_t)splitmix64_below(&rng, hi);
                cols[m][e[m]] = col;
                cpy4(vals[m] + 4 * e[m], coef + 4 * used);
                pko_fr_mul(t, coef + 4 * used, witness + 4 * (size_t)col);
                pko_fr_add(acc, acc, t);
                used++;
                e[m]++;
            }
            row_ptr[m][i + 1] = e[m];
            cpy4(dot[m], acc);
        }
        const size_t out_col = ni + 1 + i;
        cols[2][i] = (uint32_t)out_col;
        cpy4(vals[2] + 4 * i, ONE_MONT);
        row_ptr[2][i + 1] = i + 1;
        pko_fr_mul(witness + 4 * out_col, dot[0], dot[1]);
    }
    nnz_out[0] = e[0];
    nnz_out[1] = e[1];
    nnz_out[2] = nc;
    free(ka);
    free(kb);
    free(coef);
    return 0;
}

int pko_r1cs_covectors(const pko_r1cs *r1cs, const uint64_t *alpha, size_t m0, size_t len,
                       uint64_t *out) {
    const size_t nc = r1cs->num_constraints, nw = r1cs->num_witnesses;
    if (len < nw) return -1;
    uint64_t *eq = (uint64_t *)calloc(nc ? nc : 1, 32);
    if (!eq) return -2;
    memset(out, 0, 32 * 3 * len);
    pko_eq_hypercube(alpha, m0, nc, eq);
    for (int k = 0; k < 3; k++) {
        uint64_t *alph = out + 4 * len * (size_t)k;
        for (size_t row = 0; row < nc; row++)
            for (uint64_t e = r1cs->row_ptr[k][row]; e < r1cs->row_ptr[k][row + 1]; e++) {
                uint64_t tt[4];
                pko_fr_mul(tt, r1cs->vals[k] + 4 * e, eq + 4 * row);
                size_t col = r1cs->cols[k][e];
                pko_fr_add(alph + 4 * col, alph + 4 * col, tt);
            }
    }
    free(eq);
    return 0;
}

void pko_public_inputs_hash(uint64_t out[4], const uint64_t *v, size_t n) {
    static const uint64_t zero[4] = {0, 0, 0, 0};
    if (n == 0) {
        cpy4(out, zero);
        return;
    }
    if (n == 1) {
        pko_sky_compress(out, v, zero);
        return;
    }
    uint64_t h[4], t[4];
    pko_sky_compress(h, v, v + 4);
    for (size_t i = 2; i < n; i++) {
        pko_sky_compress(t, h, v + 4 * i);
        cpy4(h, t);
    }
    cpy4(out, h);
}

int pko_r1cs_statement_covectors(const pko_r1cs *r1cs, const uint64_t public_x[4],
                                 const uint64_t *alpha, size_t m0, size_t blinding_offset,
                                 size_t len, uint64_t *out) {
    const size_t np = r1cs->num_public_inputs;
    const size_t base = np ? 1 : 0, ncov = base + 4;
    if (blinding_offset + 4 * m0 > len || np + 1 > len) return -1;
    memset(out, 0, 32 * ncov * len);
    if (np) {
        uint64_t pw[4];
        cpy4(pw, ONE_MONT);
        for (size_t i = 0; i <= np; i++) {
            cpy4(out + 4 * i, pw);
            pko_fr_mul(pw, pw, public_x);
        }
    }
    int rc = pko_r1cs_covectors(r1cs, alpha, m0, len, out + 4 * len * base);
    if (rc) return rc;
    uint64_t *bl = out + 4 * len * (base + 3) + 4 * blinding_offset;
    for (size_t i = 0; i < m0; i++) {
        uint64_t pw[4];
        cpy4(pw, ONE_MONT);
        for (int k = 0; k < 4; k++) {
            cpy4(bl + 4 * (4 * i + k), pw);
            pko_fr_mul(pw, pw, alpha + 4 * i);
        }
    }
    return (int)ncov;
}

/* With whir == NULL the commitment's root alone enters the transcript and
 * the proof ends at the covector evaluations; with whir, the commitment's
 * OOD samples follow the root (pko_whir_commit_ood) and pko_whir_prove of
 * the three zero-padded covectors M^T eq(alpha) ends it, on a copy of the
 * transcript (out->transcript is the state the WHIR prover starts from). */
static int spartan_prove_impl(const pko_r1cs *r1cs, const uint64_t *witness,
                              uint64_t blinding_seed, uint64_t domain, unsigned ff, unsigned lr,
                              pko_spartan_proof *out, const pko_whir_params *whir,
                              uint64_t *whir_commit_words, uint64_t *whir_proof) {
    const size_t nc = r1cs->num_constraints, nw = r1cs->num_witnesses, w1_size = nw;
    size_t m, m0;
    pko_r1cs_sizing(nc, nw, &m, &m0);
    if (m0 > 30 || m > 28 || ff > m) return -1;
    if (whir && (whir->num_variables != m || whir->folding_factor != ff ||
                 whir->log_inv_rate != lr || whir->ood_samples > 4 ||
                 (whir->batch_size != 1 && whir->batch_size != 2)))
        return -1;
    /* whir-ZK (a WHIR batch of 2): the witness polynomial committed with a
     * blinding polynomial drawn from the indexed sampler */
    const size_t nb = whir ? whir->batch_size : 1;
    memset(out, 0, sizeof *out);
    out->m = m;
    out->m0 = m0;
    pko_transcript *t = &out->transcript;
    uint64_t dom[4] = {domain, 0, 0, 0};
    pko_transcript_init(t, dom);
    /* commit: pad, blinding coefficients at offset w1_size */
    size_t n = (size_t)1 << m;
    uint64_t *poly = (uint64_t *)calloc(n * nb, 32);
    uint64_t *g = (uint64_t *)malloc(32 * 4 * m0);
    if (!poly || !g) return -2;
    memcpy(poly, witness, 32 * nw);
    pko_sample_fr(blinding_seed, 4 * m0, g, 1);
    memcpy(poly + 4 * w1_size, g, 32 * 4 * m0);
    if (nb == 2) pko_sample_fr_indexed(blinding_seed ^ 0x243f6a8885a308d3ULL, 0, n, poly + 4 * n);
    size_t M = (size_t)1 << ff, L = n >> ff, cw_len = L << lr;
    uint64_t *cw = (uint64_t *)malloc(32 * M * nb * cw_len);
    uint8_t *layers = (uint8_t *)malloc(32 * (2 * cw_len - 1));
    if (!cw || !layers) return -2;
    int rc = pko_whir_commit(poly, n * nb, ff + (nb == 2 ? 1 : 0), lr, cw, layers);
    if (rc) return rc;
    memcpy(out->root, layers + 32 * (2 * cw_len - 2), 32);
    uint64_t ood_points[4 * 5];
    if (whir) {
        rc = pko_whir_commit_ood(whir, t, poly, out->root, whir_commit_words, ood_points);
        if (rc) return rc;
    } else {
        uint64_t root_m[4];
        memcpy(root_m, out->root, 32);
        pko_fr_to_mont(root_m, root_m);
        pko_transcript_absorb(t, root_m);
    }
    /* witness bounds (sumcheck.rs:163-179) */
    size_t n0 = (size_t)1 << m0;
    uint64_t *a = (uint64_t *)calloc(n0, 32), *b = (uint64_t *)calloc(n0, 32), *cc = (uint64_t *)calloc(n0, 32);
    if (!a || !b || !cc) return -2;
    pko_spmv(r1cs->row_ptr[0], r1cs->cols[0], r1cs->vals[0], nc, witness, a);
    pko_spmv(r1cs->row_ptr[1], r1cs->cols[1], r1cs->vals[1], nc, witness, b);
    for (size_t i = 0; i < nc; i++) pko_fr_mul(cc + 4 * i, a + 4 * i, b + 4 * i);
    /* zk sumcheck */
    rc = pko_spartan_sumcheck(t, a, b, cc, m0, g, poly, w1_size, &out->r[0][0], out->rho,
                              out->sum_g, &out->coeffs[0][0], &out->alpha[0][0], out->blinding_eval);
    free(a); free(b); free(cc); free(g);
    if (rc) return rc;
    /* eq(alpha) truncated to num_constraints, then M^T eq for A, B, C
     * (multiply_transposed_by_eq_alpha, sumcheck.rs:206-227): computed as
     * the scatter sum over the rows of M, which equals the transposed SpMV */
    uint64_t *cov = (uint64_t *)malloc(32 * 3 * n);
    if (!cov) return -2;
    /* public weights (whir_r1cs.rs:665-676): the public inputs' hash, then x */
    const size_t np = r1cs->num_public_inputs;
    if (np + 1 > nw) return -1;
    {
        uint64_t *pv = (uint64_t *)malloc(32 * (np + 1));
        if (!pv) return -2;
        memcpy(pv, witness + 4, 32 * np);
        pko_from_mont_many(pv, np);
        pko_public_inputs_hash(out->public_hash, pv, np);
        free(pv);
        uint64_t hm[4];
        pko_fr_to_mont(hm, out->public_hash);
        pko_transcript_absorb(t, hm);
    }
    pko_transcript_squeeze(t, out->public_x);
    if ((rc = pko_r1cs_covectors(r1cs, &out->alpha[0][0], m0, n, cov))) return rc;
    for (int k = 0; k < 3; k++) {
        /* create_weights_and_evaluations (:623-642): dot over the padded prefix */
        pko_dot(out->evals[k], cov + 4 * n * (size_t)k, poly, nw);
        pko_transcript_absorb(t, out->evals[k]);
    }
    if (np) { /* compute_public_weight_evaluation (:654-663), then its message (:281) */
        uint64_t pw[4], x[4];
        cpy4(pw, ONE_MONT);
        memset(out->public_eval, 0, 32);
        for (size_t i = 0; i <= np; i++) {
            pko_fr_mul(x, pw, poly + 4 * i);
            pko_fr_add(out->public_eval, out->public_eval, x);
            pko_fr_mul(pw, pw, out->public_x);
        }
        pko_transcript_absorb(t, out->public_eval);
    }
    if (whir) {
        /* the statements [public?, A, B, C, blinding] (prove_from_alphas, :258-301) */
        uint64_t *stmts = (uint64_t *)malloc(32 * 5 * n);
        if (!stmts) return -2;
        int ncov = pko_r1cs_statement_covectors(r1cs, out->public_x, &out->alpha[0][0], m0, w1_size,
                                                n, stmts);
        pko_transcript tw = *t;
        rc = ncov < 0 ? ncov
                      : pko_whir_prove(whir, &tw, poly, cw, layers, whir_commit_words, ood_points,
                                       stmts, (size_t)ncov, whir_proof);
        free(stmts);
    }
    free(cov); free(poly); free(cw); free(layers);
    return rc;
}

int pko_spartan_prove(const pko_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                      uint64_t domain, unsigned ff, unsigned lr, pko_spartan_proof *out) {
    return spartan_prove_impl(r1cs, witness, blinding_seed, domain, ff, lr, out, NULL, NULL, NULL);
}

int pko_prove_r1cs(const pko_r1cs *r1cs, const uint64_t *witness, uint64_t blinding_seed,
                   uint64_t domain, const pko_whir_params *whir, pko_spartan_proof *out,
                   uint64_t *whir_commit_words, uint64_t *whir_proof) {
    if (!whir || !whir_commit_words || !whir_proof) return -1;
    return spartan_prove_impl(r1cs, witness, blinding_seed, domain, whir->folding_factor,
                              whir->log_inv_rate, out, whir, whir_commit_words, whir_proof);
}

/* ----------------------------------------------------------------------- */
/* Two commitments: R1CS with verifier challenges                          */
/* ----------------------------------------------------------------------- */
void pko_r1cs_sizing_split(size_t num_constraints, size_t num_witnesses, size_t w1_size,
                           size_t *m_out, size_t *m0_out) {
    /* new_for_r1cs (r1cs-compiler/src/whir_r1cs.rs:48-92) */
    const size_t m1 = ceil_log2(w1_size), m2 = ceil_log2(num_witnesses - w1_size);
    size_t m = m1 > m2 ? m1 : m2, m0 = ceil_log2(num_constraints);
    if (m < 13) m = 13;
    if (m0 < 1) m0 = 1;
    if (((size_t)1 << m) - w1_size < 4 * m0) m++;
    *m_out = m;
    *m0_out = m0;
}

/* One part's commitment (whir_r1cs.rs commit, :82-140): its nvals values
 * padded to n, g (4 m0 Fr) at g_offset when given, with batch 2 the mask
 * polynomial in the second half; RS encode + tree, then the OOD samples. */
static int dual_commit(const pko_whir_params *whir, pko_transcript *t, const uint64_t *vals,
                       size_t nvals, const uint64_t *g, size_t g_len, size_t g_offset,
                       uint64_t mask_seed, uint64_t *poly, uint64_t *cw, uint8_t *layers,
                       uint8_t root[32], uint64_t *commit_words, uint64_t *ood_points) {
    const size_t n = (size_t)1 << whir->num_variables, nb = whir->batch_size;
    const unsigned ff = whir->folding_factor, lr = whir->log_inv_rate;
    memset(poly, 0, 32 * n * nb);
    if (nvals) memcpy(poly, vals, 32 * nvals);
    if (g) memcpy(poly + 4 * g_offset, g, 32 * g_len);
    if (nb == 2) pko_sample_fr_indexed(mask_seed, 0, n, poly + 4 * n);
    const size_t cw_len = (n >> ff) << lr;
    int rc = pko_whir_commit(poly, n * nb, ff + (nb == 2 ? 1 : 0), lr, cw, layers);
    if (rc) return rc;
    memcpy(root, layers + 32 * (2 * cw_len - 2), 32);
    return pko_whir_commit_ood(whir, t, poly, root, commit_words, ood_points);
}

int pko_prove_r1cs_dual(const pko_r1cs *r1cs, size_t w1_size, const size_t *offs, size_t nchal,
                        uint64_t *witness, pko_w2_solver solve, void *ctx,
                        uint64_t blinding_seed, uint64_t domain, const pko_whir_params *whir,
                        pko_dual_proof *out, uint64_t *challenges, uint64_t *commit_words1,
                        uint64_t *commit_words2, uint64_t *proof1, uint64_t *proof2) {
    const size_t nc = r1cs->num_constraints, nw = r1cs->num_witnesses;
    const size_t np = r1cs->num_public_inputs;
    if (!whir || !solve || w1_size < np + 1 || w1_size > nw) return -1;
    size_t m, m0;
    pko_r1cs_sizing_split(nc, nw, w1_size, &m, &m0);
    if (m0 > 30 || m > 28 || whir->num_variables != m || whir->folding_factor > m ||
        whir->ood_samples > 4 || (whir->batch_size != 1 && whir->batch_size != 2))
        return -1;
    const size_t n = (size_t)1 << m, nb = whir->batch_size, w2_size = nw - w1_size;
    for (size_t j = 0; j < nchal; j++)
        if (offs[j] >= n) return -1; /* SparseCovector::new (prefix_covector.rs:257-266) */
    memset(out, 0, sizeof *out);
    pko_spartan_proof *sp = &out->spartan;
    sp->m = m;
    sp->m0 = m0;
    pko_transcript *t = &sp->transcript;
    const uint64_t dom[4] = {domain, 0, 0, 0};
    pko_transcript_init(t, dom);

    const size_t cw_len = (n >> whir->folding_factor) << whir->log_inv_rate;
    const size_t cw_fr = ((size_t)1 << whir->folding_factor) * nb * cw_len;
    uint64_t *poly1 = malloc(32 * n * nb), *poly2 = malloc(32 * n * nb);
    uint64_t *cw1 = malloc(32 * cw_fr), *cw2 = malloc(32 * cw_fr);
    uint8_t *lay1 = malloc(32 * (2 * cw_len - 1)), *lay2 = malloc(32 * (2 * cw_len - 1));
    uint64_t *g = malloc(32 * 4 * m0);
    size_t n0 = (size_t)1 << m0;
    uint64_t *a = calloc(n0, 32), *b = calloc(n0, 32), *cc = calloc(n0, 32);
    uint64_t *cov = malloc(32 * 3 * (nw ? nw : 1));
    uint64_t *st1 = malloc(32 * 5 * n), *st2 = malloc(32 * 4 * n);
    uint64_t ood1[4 * 5], ood2[4 * 5];
    int rc = -2;
    if (!poly1 || !poly2 || !cw1 || !cw2 || !lay1 || !lay2 || !g || !a || !b || !cc || !cov ||
        !st1 || !st2)
        goto done;

    /* commit w1 with the blinding univariates at w1_size (lib.rs:184-187) */
    pko_sample_fr(blinding_seed, 4 * m0, g, 1);
    rc = dual_commit(whir, t, witness, w1_size, g, 4 * m0, w1_size,
                     blinding_seed ^ 0x243f6a8885a308d3ULL, poly1, cw1, lay1, sp->root,
                     commit_words1, ood1);
    if (rc) goto done;
    /* the challenges (WitnessBuilder::Challenge, witness_builder.rs:167-170),
     * then the caller's solve of w2 and its commitment (lib.rs:189-217) */
    for (size_t j = 0; j < nchal; j++) pko_transcript_squeeze(t, challenges + 4 * j);
    solve(ctx, challenges, nchal, witness);
    rc = dual_commit(whir, t, witness + 4 * w1_size, w2_size, NULL, 0, 0,
                     blinding_seed ^ 0x13198a2e03707344ULL, poly2, cw2, lay2, out->root2,
                     commit_words2, ood2);
    if (rc) goto done;

    /* witness bounds over the whole witness, the zk sumcheck with w1's
     * blinding (prove_noir, whir_r1cs.rs:143-187) */
    pko_spmv(r1cs->row_ptr[0], r1cs->cols[0], r1cs->vals[0], nc, witness, a);
    pko_spmv(r1cs->row_ptr[1], r1cs->cols[1], r1cs->vals[1], nc, witness, b);
    for (size_t i = 0; i < nc; i++) pko_fr_mul(cc + 4 * i, a + 4 * i, b + 4 * i);
    rc = pko_spartan_sumcheck(t, a, b, cc, m0, g, poly1, w1_size, &sp->r[0][0], sp->rho,
                              sp->sum_g, &sp->coeffs[0][0], &sp->alpha[0][0], sp->blinding_eval);
    if (rc) goto done;
    /* get_public_weights (:665-676) */
    {
        uint64_t *pv = malloc(32 * (np + 1)), hm[4];
        if (!pv) { rc = -2; goto done; }
        memcpy(pv, witness + 4, 32 * np);
        pko_from_mont_many(pv, np);
        pko_public_inputs_hash(sp->public_hash, pv, np);
        free(pv);
        pko_fr_to_mont(hm, sp->public_hash);
        pko_transcript_absorb(t, hm);
    }
    pko_transcript_squeeze(t, sp->public_x);
    /* alphas split at w1_size (:311-326); compute_alpha_evals (prefix_covector.rs:212-223) */
    if ((rc = pko_r1cs_covectors(r1cs, &sp->alpha[0][0], m0, nw, cov))) goto done;
    for (int k = 0; k < 3; k++) pko_dot(sp->evals[k], cov + 4 * nw * (size_t)k, poly1, w1_size);
    for (int k = 0; k < 3; k++)
        pko_dot(out->evals2[k], cov + 4 * (nw * (size_t)k + w1_size), poly2, w2_size);
    for (int k = 0; k < 3; k++) pko_transcript_absorb(t, sp->evals[k]);
    for (int k = 0; k < 3; k++) pko_transcript_absorb(t, out->evals2[k]);
    uint64_t pw[4], x[4];
    if (np) { /* compute_public_eval (prefix_covector.rs:226-240) on w1 */
        cpy4(pw, ONE_MONT);
        for (size_t i = 0; i <= np; i++) {
            pko_fr_mul(x, pw, poly1 + 4 * i);
            pko_fr_add(sp->public_eval, sp->public_eval, x);
            pko_fr_mul(pw, pw, sp->public_x);
        }
        pko_transcript_absorb(t, sp->public_eval);
    }
    if (nchal) { /* compute_challenge_eval (prefix_covector.rs:326-338) on w2 */
        cpy4(pw, ONE_MONT);
        for (size_t j = 0; j < nchal; j++) {
            pko_fr_mul(x, pw, poly2 + 4 * offs[j]);
            pko_fr_add(out->challenge_eval, out->challenge_eval, x);
            pko_fr_mul(pw, pw, sp->public_x);
        }
        pko_transcript_absorb(t, out->challenge_eval);
    }

    /* w1's statements: the public weight first (make_public_weight, :350-356),
     * the alphas restricted to w1, the blinding covector expand_powers::<4>(alpha)
     * at w1_size (the whole witness may be longer than 2^m: each part is not) */
    const size_t base = np ? 1 : 0, ncov1 = base + 4, ncov2 = 3 + (nchal ? 1 : 0);
    memset(st1, 0, 32 * ncov1 * n);
    if (np) {
        cpy4(pw, ONE_MONT);
        for (size_t i = 0; i <= np; i++) {
            cpy4(st1 + 4 * i, pw);
            pko_fr_mul(pw, pw, sp->public_x);
        }
    }
    for (int k = 0; k < 3; k++)
        memcpy(st1 + 4 * n * (base + (size_t)k), cov + 4 * nw * (size_t)k, 32 * w1_size);
    for (size_t i = 0; i < m0; i++) {
        uint64_t *bl = st1 + 4 * (n * (base + 3) + w1_size + 4 * i);
        cpy4(pw, ONE_MONT);
        for (int q = 0; q < 4; q++) {
            cpy4(bl + 4 * q, pw);
            pko_fr_mul(pw, pw, sp->alpha[i]);
        }
    }
    /* w2's statements: the alphas restricted to w2, the challenge weight
     * (make_challenge_weight, prefix_covector.rs:311-323; SparseCovector
     * accumulates, so repeated offsets add) */
    memset(st2, 0, 32 * ncov2 * n);
    for (int k = 0; k < 3; k++)
        memcpy(st2 + 4 * n * (size_t)k, cov + 4 * (nw * (size_t)k + w1_size), 32 * w2_size);
    if (nchal) {
        cpy4(pw, ONE_MONT);
        for (size_t j = 0; j < nchal; j++) {
            uint64_t *e = st2 + 4 * (3 * n + offs[j]);
            pko_fr_add(e, e, pw);
            pko_fr_mul(pw, pw, sp->public_x);
        }
    }
    {
        pko_transcript tw = *t;
        rc = pko_whir_prove(whir, &tw, poly1, cw1, lay1, commit_words1, ood1, st1, ncov1, proof1);
        if (!rc)
            rc = pko_whir_prove(whir, &tw, poly2, cw2, lay2, commit_words2, ood2, st2, ncov2,
                                proof2);
    }
done:
    free(poly1); free(poly2); free(cw1); free(cw2); free(lay1); free(lay2); free(g);
    free(a); free(b); free(cc); free(cov); free(st1); free(st2);
    return rc;
}

int pko_synthetic_r1cs_dual(uint64_t seed, size_t nc1, size_t ni, size_t nchal, size_t rows2,
                            uint64_t *row_ptr[3], uint32_t *cols[3], uint64_t *vals[3],
                            size_t nnz_out[3], uint64_t *witness, size_t *offs) {
    const size_t w1 = 1 + ni + nc1, w2 = nchal + rows2;
    if (w1 + w2 >= ((size_t)1 << 32)) return -1;
    int rc = pko_synthetic_r1cs(seed, nc1, ni, row_ptr, cols, vals, nnz_out, witness);
    if (rc) return rc;
    memset(witness + 4 * w1, 0, 32 * w2);
    /* w2's layout: challenges spread at multiples of the stride, products
     * at the remaining offsets in order */
    const size_t stride = nchal ? w2 / nchal : 0;
    for (size_t j = 0; j < nchal; j++) offs[j] = j * stride;
    uint64_t rng = seed ^ 0xd1b54a32d192ed03ULL;
    uint64_t *coef = malloc(32 * 2 * (rows2 ? rows2 : 1));
    if (!coef) return -2;
    pko_sample_fr(seed + 2, 2 * rows2, coef, 1);
    size_t e[2] = {nnz_out[0], nnz_out[1]}, used = 0, next = 0, j = 0;
    for (size_t i = 0; i < rows2; i++) {
        const size_t row = nc1 + i;
        /* A: the challenge (or the constant) with coefficient 1 */
        cols[0][e[0]] = (uint32_t)(nchal ? w1 + offs[i % nchal] : 0);
        cpy4(vals[0] + 4 * e[0], ONE_MONT);
        e[0]++;
        row_ptr[0][row + 1] = e[0];
        /* B: 1-2 uniform w1 columns */
        const int kb = 1 + (int)splitmix64_below(&rng, 2);
        for (int q = 0; q < kb; q++) {
            cols[1][e[1]] = (uint32_t)splitmix64_below(&rng, w1);
            cpy4(vals[1] + 4 * e[1], coef + 4 * used++);
            e[1]++;
        }
        row_ptr[1][row + 1] = e[1];
        /* C: the next offset that holds no challenge */
        while (j < nchal && offs[j] == next) { next++; j++; }
        cols[2][row] = (uint32_t)(w1 + next);
        cpy4(vals[2] + 4 * row, ONE_MONT);
        row_ptr[2][row + 1] = row + 1;
        next++;
    }
    free(coef);
    nnz_out[0] = e[0];
    nnz_out[1] = e[1];
    nnz_out[2] = nc1 + rows2;
    return 0;
}

void pko_synthetic_dual_solve(void *ctx, const uint64_t *chal, size_t nchal, uint64_t *w) {
    const pko_synthetic_dual *d = (const pko_synthetic_dual *)ctx;
    const pko_r1cs *r = d->r1cs;
    for (size_t j = 0; j < nchal; j++) cpy4(w + 4 * (d->w1_size + d->challenge_offsets[j]), chal + 4 * j);
    for (size_t row = d->first_row; row < r->num_constraints; row++) {
        uint64_t dot[2][4], t[4];
        for (int k = 0; k < 2; k++) {
            memset(dot[k], 0, 32);
            for (uint64_t e = r->row_ptr[k][row]; e < r->row_ptr[k][row + 1]; e++) {
                pko_fr_mul(t, r->vals[k] + 4 * e, w + 4 * (size_t)r->cols[k][e]);
                pko_fr_add(dot[k], dot[k], t);
            }
        }
        pko_fr_mul(w + 4 * (size_t)r->cols[2][r->row_ptr[2][row]], dot[0], dot[1]);
    }
}

/* ======================================================================= */
/* Poseidon2, t = 4, rf = 8, rp = 56 (poseidon2/src/permutation.rs)         */
/* ======================================================================= */
static void p2_sbox(uint64_t x[4]) { /* x^5, :86-89 */
    uint64_t s[4];
    pko_fr_mul(s, x, x);
    pko_fr_mul(s, s, s);
    pko_fr_mul(x, s, x);
}

static void p2_ext(uint64_t st[16]) { /* matrix_multiplication_4x4, :101-120 */
    uint64_t t0[4], t1[4], t2[4], t3[4], t4[4], t5[4], t6[4], t7[4];
    pko_fr_add(t0, st, st + 4);
    pko_fr_add(t1, st + 8, st + 12);
    pko_fr_add(t2, st + 4, st + 4);
    pko_fr_add(t2, t2, t1);
    pko_fr_add(t3, st + 12, st + 12);
    pko_fr_add(t3, t3, t0);
    pko_fr_add(t4, t1, t1);
    pko_fr_add(t4, t4, t4);
    pko_fr_add(t4, t4, t3);
    pko_fr_add(t5, t0, t0);
    pko_fr_add(t5, t5, t5);
    pko_fr_add(t5, t5, t2);
    pko_fr_add(t6, t3, t5);
    pko_fr_add(t7, t2, t4);
    cpy4(st, t6);
    cpy4(st + 4, t5);
    cpy4(st + 8, t7);
    cpy4(st + 12, t4);
}

static void p2_int(uint64_t st[16]) { /* internal_m_multiplication, :122-127 */
    uint64_t sum[4] = {0, 0, 0, 0}, t[4];
    for (int i = 0; i < 4; i++) pko_fr_add(sum, sum, st + 4 * i);
    for (int i = 0; i < 4; i++) {
        pko_fr_mul(t, st + 4 * i, POSEIDON2_T4_DIAG_MONT[i]);
        pko_fr_add(st + 4 * i, t, sum);
    }
}

void pko_poseidon2_permutation(uint64_t st[16]) { /* permutation, :134-167 */
    p2_ext(st);
    for (int r = 0; r < 64; r++) {
        if (r < 4 || r >= 60) {
            for (int i = 0; i < 4; i++) {
                pko_fr_add(st + 4 * i, st + 4 * i, POSEIDON2_T4_RC_MONT[r][i]);
                p2_sbox(st + 4 * i);
            }
            p2_ext(st);
        } else {
            pko_fr_add(st, st, POSEIDON2_T4_RC_MONT[r][0]);
            p2_sbox(st);
            p2_int(st);
        }
    }
}

/* poseidon2_hash (poseidon2/src/hash.rs:17-47): rate 3, IV = len * 2^64 in lane 3. */
void pko_poseidon2_hash(uint64_t out[4], const uint64_t *inputs, size_t n) {
    uint64_t st[16] = {0}, cache[12] = {0};
    uint64_t two64[4] = {0, 1, 0, 0}, lenv[4] = {n, 0, 0, 0};
    pko_fr_to_mont(two64, two64);
    pko_fr_to_mont(lenv, lenv);
    pko_fr_mul(st + 12, lenv, two64);
    size_t cs = 0;
    for (size_t k = 0; k < n; k++) {
        if (cs == 3) {
            for (int i = 0; i < 3; i++) pko_fr_add(st + 4 * i, st + 4 * i, cache + 4 * i);
            memset(cache, 0, sizeof cache);
            cs = 0;
            pko_poseidon2_permutation(st);
        }
        cpy4(cache + 4 * cs, inputs + 4 * k);
        cs++;
    }
    for (size_t i = 0; i < cs; i++) pko_fr_add(st + 4 * i, st + 4 * i, cache + 4 * i);
    pko_poseidon2_permutation(st);
    cpy4(out, st);
}


/* ======================================================================= */
/* WHIR prove-round building blocks (conventions of the reference's Go      */
/* WHIR verifier: recursive-verifier/app/utilities/utilities.go,            */
/* recursive-verifier/app/circuit/whir_utilities.go)                        */
/* ======================================================================= */
/* MultivarPoly (utilities.go:16-23) splits the coefficients in halves on the
 * last variable, so row entry j carries prod_t alpha[t]^(bit t of j). */
void pko_multilinear_weights(uint64_t *w, const uint64_t *alpha, unsigned k) {
    size_t m = (size_t)1 << k;
    cpy4(w, ONE_MONT);
    for (unsigned t = 0; t < k; t++) {
        size_t half = (size_t)1 << t;
        for (size_t j = 0; j < half; j++) pko_fr_mul(w + 4 * (j + half), w + 4 * j, alpha + 4 * t);
    }
    (void)m;
}

int pko_whir_fold_coeffs(const uint64_t *coeffs, size_t n, unsigned k, const uint64_t *alpha,
                         uint64_t *out) {
    if (k > 16 || !is_pow2(n) || n < ((size_t)1 << k)) return -1;
    size_t m = (size_t)1 << k, L = n >> k;
    uint64_t *w = (uint64_t *)malloc(32 * m);
    if (!w) return -2;
    pko_multilinear_weights(w, alpha, k);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < L; i++) {
        uint64_t acc[4] = {0, 0, 0, 0}, t[4];
        for (size_t j = 0; j < m; j++) {
            pko_fr_mul(t, w + 4 * j, coeffs + 4 * (j * L + i));
            pko_fr_add(acc, acc, t);
        }
        cpy4(out + 4 * i, acc);
    }
    free(w);
    return 0;
}

/* computeFold (whir_utilities.go:182-188): MultivarPoly of each row. */
int pko_whir_fold_rows(const uint64_t *rows, size_t nrows, unsigned k, const uint64_t *alpha,
                       uint64_t *out) {
    if (k > 16) return -1;
    size_t m = (size_t)1 << k;
    uint64_t *w = (uint64_t *)malloc(32 * m);
    if (!w) return -2;
    pko_multilinear_weights(w, alpha, k);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nrows; i++) {
        uint64_t acc[4] = {0, 0, 0, 0}, t[4];
        for (size_t j = 0; j < m; j++) {
            pko_fr_mul(t, w + 4 * j, rows + 4 * (i * m + j));
            pko_fr_add(acc, acc, t);
        }
        cpy4(out + 4 * i, acc);
    }
    free(w);
    return 0;
}

/* UnivarPoly (utilities.go:25-39): Horner from the top coefficient. */
void pko_poly_eval(uint64_t out[4], const uint64_t *coeffs, size_t n, const uint64_t z[4]) {
    uint64_t acc[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < n; i++) {
        pko_fr_mul(acc, acc, z);
        pko_fr_add(acc, acc, coeffs + 4 * (n - 1 - i));
    }
    cpy4(out, acc);
}

/* ExpandFromUnivariate (utilities.go:183-191). */
void pko_expand_from_univariate(uint64_t *out, const uint64_t z[4], size_t n) {
    uint64_t acc[4];
    cpy4(acc, z);
    for (size_t i = 0; i < n; i++) {
        cpy4(out + 4 * (n - 1 - i), acc);
        pko_fr_mul(acc, acc, acc);
    }
}

int pko_merkle_open(const uint8_t *layers, size_t num_leaves, uint64_t idx, uint8_t *path) {
    if (!is_pow2(num_leaves) || idx >= num_leaves) return -1;
    int depth = log2_exact(num_leaves);
    size_t off = 0, width = num_leaves;
    for (int l = 0; l < depth; l++) {
        memcpy(path + 32 * l, layers + 32 * (off + ((idx >> l) ^ 1)), 32);
        off += width;
        width >>= 1;
    }
    return 0;
}

/* verifyMerkleTreeProofs (whir_utilities.go:14-47) for one leaf; the
 * sibling of the leaf hash is path[0], the auth path the rest. */
int pko_merkle_verify(const uint64_t *leaf_canonical, size_t fr_per_leaf, uint64_t idx,
                      const uint8_t *path, size_t depth, const uint8_t root[32]) {
    uint64_t h[4], l[4], r[4], s[4];
    if (fr_per_leaf == 0) return 0;
    cpy4(h, leaf_canonical);
    for (size_t x = 1; x < fr_per_leaf; x++) {
        pko_sky_compress(l, h, leaf_canonical + 4 * x);
        cpy4(h, l);
    }
    for (size_t lev = 0; lev < depth; lev++) {
        memcpy(s, path + 32 * lev, 32);
        if ((idx >> lev) & 1) { cpy4(l, s); cpy4(r, h); }
        else { cpy4(l, h); cpy4(r, s); }
        pko_sky_compress(h, l, r);
    }
    return memcmp(h, root, 32) == 0;
}

/* getStirChallenges (whir_utilities.go:49-79) for a power-of-two folded
 * domain. */
void pko_stir_indices(const uint8_t *bytes, size_t folded_domain_size, size_t nq, uint64_t *out) {
    int bits = log2_exact(folded_domain_size);
    size_t nbytes = (size_t)(bits + 7) / 8;
    for (size_t i = 0; i < nq; i++) {
        uint64_t v = 0;
        for (size_t j = 0; j < nbytes; j++) v = (v << 8) | bytes[i * nbytes + j];
        out[i] = bits >= 64 ? v : (v & (((uint64_t)1 << bits) - 1));
    }
}

int pko_whir_sumcheck_round(uint64_t *f, uint64_t *w, size_t size, const uint64_t *fold,
                            uint64_t out[12]) {
    if (!is_pow2(size) || size < 2 || (fold && size < 4)) return -1;
    if (fold) {
        size_t h = size / 2;
        uint64_t *tabs[2] = {f, w};
        for (int k = 0; k < 2; k++) {
            uint64_t *t = tabs[k];
#pragma omp parallel for schedule(static)
            for (size_t i = 0; i < h; i++) {
                uint64_t d[4];
                pko_fr_sub(d, t + 4 * (i + h), t + 4 * i);
                pko_fr_mul(d, fold, d);
                pko_fr_add(t + 4 * i, t + 4 * i, d);
            }
        }
        size = h;
    }
    size_t half = size / 2;
    uint64_t h0[4] = {0, 0, 0, 0}, h1[4] = {0, 0, 0, 0}, h2[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < half; i++) {
        uint64_t t[4], a[4], b[4];
        pko_fr_mul(t, f + 4 * i, w + 4 * i);
        pko_fr_add(h0, h0, t);
        pko_fr_mul(t, f + 4 * (i + half), w + 4 * (i + half));
        pko_fr_add(h1, h1, t);
        /* value at X = 2: 2*hi - lo */
        pko_fr_add(a, f + 4 * (i + half), f + 4 * (i + half));
        pko_fr_sub(a, a, f + 4 * i);
        pko_fr_add(b, w + 4 * (i + half), w + 4 * (i + half));
        pko_fr_sub(b, b, w + 4 * i);
        pko_fr_mul(t, a, b);
        pko_fr_add(h2, h2, t);
    }
    cpy4(out, h0);
    cpy4(out + 4, h1);
    cpy4(out + 8, h2);
    return 0;
}

int pko_eq_accumulate(uint64_t *w, size_t nv, const uint64_t *points, const uint64_t *coeffs,
                      size_t npts) {
    if (nv >= 40) return -1;
    size_t n = (size_t)1 << nv;
    uint64_t *eq = (uint64_t *)malloc(32 * n);
    if (!eq) return -2;
    for (size_t j = 0; j < npts; j++) {
        pko_eq_hypercube(points + 4 * nv * j, nv, n, eq);
#pragma omp parallel for schedule(static)
        for (size_t b = 0; b < n; b++) {
            uint64_t t[4];
            pko_fr_mul(t, coeffs + 4 * j, eq + 4 * b);
            pko_fr_add(w + 4 * b, w + 4 * b, t);
        }
    }
    free(eq);
    return 0;
}
