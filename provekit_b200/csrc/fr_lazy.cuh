// fr_lazy.cuh -- exact sums of BN254 Fr Montgomery products on the FP64
// pipe, reduced once per sum.
//
// A sum S = sum_k a_k b_k of products of Montgomery-form values is needed
// reduced only once.  The products are accumulated as exact unreduced
// integers in binary64 columns and one Montgomery reduction follows,
// instead of one per product (fr_f64.cuh): per term 144 digit products and
// 24 digit conversions instead of ~350 binary64 instructions.
//
// Digits are 22 bits (12 per operand, 264 >= 256 bits), held as exact
// doubles:
//  * a digit product is < 2^44 and a column receives at most 12 of them per
//    term, so a term adds < 12 * 2^44 < 2^47.6 to a column;
//  * carry() splits every column into its low 22 bits and the rest and moves
//    the rest one column up, all columns at once (no ripple): a column is
//    then < 2^22 + 2^31; kCarryEvery = 32 terms between carries keep every
//    column below 2^31.1 + 32 * 2^47.6 < 2^52.6 < 2^53, so every fma is exact;
//  * finish() ripples the carries into 24 exact 22-bit digits of T = S and
//    divides by 2^264 in twelve Montgomery steps: p = 1 mod 2^28 makes
//    -p^-1 = -1 mod 2^22, so the step's digit for the low column T_s is
//    (-T_s) mod 2^22, read off a round-up add of 2^74 (ulp 2^22), and
//    T_s + q = u carries u / 2^22 up.  The quotient V = (T + Q p) / 2^264 <
//    T / 2^264 + p; with every operand < p, T < K p^2 for K terms, and V <
//    (K p / 2^264 + 1) p < 2p for K <= kMaxTerms (p / 2^264 < 1 / 1354), so
//    one conditional subtraction finishes.
// The result is S * 2^-264 mod p: callers fold the missing 2^8 into an
// operand (a coefficient times 2^8) or multiply the result by kMont2e8
// (2^8 in Montgomery form) with one Montgomery product.
// Every constant is a power of two or a 22-bit digit of p; nothing depends
// on the rounding of an inexact operation.
#pragma once
#include "fr.cuh"

namespace pk {
namespace lazy {

constexpr int kD = 12;           // 22-bit digits per operand
constexpr int kCols = 24;        // product columns 0..22, carry column 23
constexpr int kCarryEvery = 32;  // terms between carry() calls
constexpr int kMaxTerms = 1024;  // terms per finish() (operands < p)

constexpr double kTwo52 = 4503599627370496.0;         // 2^52
constexpr double kTwo74 = 18889465931478580854784.0;  // 2^74 (ulp 2^22)
constexpr double kInv22 = 1.0 / 4194304.0;            // 2^-22

// 2^8 in Montgomery form (2^264 mod p), 64-bit limbs
constexpr uint64_t kMont2e8[4] = {0xf6e31f8c9ffffab6ULL, 0x5d7570ac31329faeULL,
                                  0x276f48b709e2a349ULL, 0x0d791464ef86e357ULL};

// p in 22-bit digits, least significant first (digit 0 is 1).
__device__ __forceinline__ double pdig(int j) {
  constexpr double P[kD] = {1.0,       1462208.0, 1326623.0, 3038244.0, 2639993.0, 3449039.0,
                            1578373.0, 1142176.0, 2734160.0, 312960.0,  321326.0,  3097.0};
  return P[j];
}

__device__ __forceinline__ double dbl(uint32_t v) {
  return __hiloint2double(0x43300000, (int)v) - kTwo52;
}

// the twelve 22-bit digits of a 256-bit value, least significant first
__device__ __forceinline__ void digits(const Fr& a, double* A) {
  const uint32_t M = 0x3FFFFFu;
  A[0] = dbl(a.v[0] & M);                                 // bits   0..21
  A[1] = dbl(__funnelshift_r(a.v[0], a.v[1], 22) & M);   // bits  22..43
  A[2] = dbl(__funnelshift_r(a.v[1], a.v[2], 12) & M);   // bits  44..65
  A[3] = dbl(__funnelshift_r(a.v[2], a.v[3], 2) & M);    // bits  66..87
  A[4] = dbl(__funnelshift_r(a.v[2], a.v[3], 24) & M);   // bits  88..109
  A[5] = dbl(__funnelshift_r(a.v[3], a.v[4], 14) & M);   // bits 110..131
  A[6] = dbl(__funnelshift_r(a.v[4], a.v[5], 4) & M);    // bits 132..153
  A[7] = dbl(__funnelshift_r(a.v[4], a.v[5], 26) & M);   // bits 154..175
  A[8] = dbl(__funnelshift_r(a.v[5], a.v[6], 16) & M);   // bits 176..197
  A[9] = dbl(__funnelshift_r(a.v[6], a.v[7], 6) & M);    // bits 198..219
  A[10] = dbl(__funnelshift_r(a.v[6], a.v[7], 28) & M);  // bits 220..241
  A[11] = dbl(a.v[7] >> 18);                              // bits 242..255
}

struct Acc {
  double c[kCols];

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < kCols; i++) c[i] = 0.0;
  }

  // c += A * B (digit forms)
  __device__ __forceinline__ void mac(const double* A, const double* B) {
#pragma unroll
    for (int i = 0; i < kD; i++)
#pragma unroll
      for (int j = 0; j < kD; j++) c[i + j] = fma(A[i], B[j], c[i + j]);
  }

  __device__ __forceinline__ void mac(const Fr& a, const Fr& b) {
    double A[kD], B[kD];
    digits(a, A);
    digits(b, B);
    mac(A, B);
  }

  // every column to its low 22 bits plus the carry of the column below
  __device__ __forceinline__ void carry() {
    double hi[kCols];
#pragma unroll
    for (int i = 0; i < kCols; i++) {
      const double w = __dadd_rz(c[i], kTwo74) - kTwo74;  // floor(c / 2^22) * 2^22
      hi[i] = w * kInv22;
      c[i] -= w;
    }
#pragma unroll
    for (int i = 1; i < kCols; i++) c[i] += hi[i - 1];
  }

  // sum * 2^-264 mod p, fully reduced (at most kMaxTerms terms, operands < p)
  __device__ __forceinline__ Fr finish() const {
    double T[kCols];
    double x = 0.0;
#pragma unroll
    for (int i = 0; i < kCols; i++) {  // exact 22-bit digits (ripple)
      x += c[i];
      const double w = __dadd_rz(x, kTwo74) - kTwo74;
      T[i] = x - w;
      x = w * kInv22;
    }
#pragma unroll
    for (int s = 0; s < kD; s++) {  // twelve 22-bit Montgomery steps
      const double u = __dadd_ru(T[s], kTwo74) - kTwo74;
      const double q = u - T[s];
      T[s + 1] = fma(u, kInv22, T[s + 1]);
#pragma unroll
      for (int j = 1; j < kD; j++) T[s + j] = fma(q, pdig(j), T[s + j]);
    }
    // V = T[12..23] < 2p < 2^255 as exact 22-bit digits, then 32-bit limbs
    uint32_t d[kD];
    x = 0.0;
#pragma unroll
    for (int i = 0; i < kD; i++) {
      x += T[kD + i];
      const double w = __dadd_rz(x, kTwo74) - kTwo74;
      d[i] = (uint32_t)__double2loint((x - w) + kTwo52);
      x = w * kInv22;
    }
    Fr r;
    r.v[0] = d[0] | (d[1] << 22);
    r.v[1] = (d[1] >> 10) | (d[2] << 12);
    r.v[2] = (d[2] >> 20) | (d[3] << 2) | (d[4] << 24);
    r.v[3] = (d[4] >> 8) | (d[5] << 14);
    r.v[4] = (d[5] >> 18) | (d[6] << 4) | (d[7] << 26);
    r.v[5] = (d[7] >> 6) | (d[8] << 16);
    r.v[6] = (d[8] >> 16) | (d[9] << 6) | (d[10] << 28);
    r.v[7] = (d[10] >> 4) | (d[11] << 18);
    return fr_reduce_once(r);
  }
};

// kMont2e8 as device 32-bit limbs
__device__ __forceinline__ Fr mont_2e8() {
  Fr r;
  r.v[0] = 0x9ffffab6u; r.v[1] = 0xf6e31f8cu; r.v[2] = 0x31329faeu; r.v[3] = 0x5d7570acu;
  r.v[4] = 0x09e2a349u; r.v[5] = 0x276f48b7u; r.v[6] = 0xef86e357u; r.v[7] = 0x0d791464u;
  return r;
}

}  // namespace lazy
}  // namespace pk
