// BN254 Fr Montgomery product and square on the FP64 (DFMA) pipe.
//
// B200 issues double-precision FMAs at the same rate as 32-bit integer
// multiply-adds, and the two share that throughput (mixing them gains
// nothing), so the form that is faster on its own wins; on B200 that is this
// one (352 binary64 instructions per product, 296 per square).  These routines compute exactly the same integers as fr_mul / fr_sqr
// (a*b*2^-256 mod p, fully reduced), but do their products in binary64.  They follow the idea of Emmart, Zheng and Weems,
// "Faster Modular Exponentiation Using Double Precision Floating Point
// Arithmetic on the GPU" (ARITH 2018), with a digit size chosen so that no
// product ever needs splitting:
//
//  * operands are 11 digits of 24 bits held as doubles (exact integers);
//  * a digit product is < 2^48, and a column never holds more than 11 operand
//    products + 10 reduction products + one carry (< 2^29), so every
//    column sum stays below 21 * 2^48 + 2^29 < 2^53: each fma is exact;
//  * p = 1 mod 2^28, so -p^-1 = -1 mod 2^24 and the Montgomery digit of a
//    column T0 is simply (-T0) mod 2^24.  A round-up add of 2^76 (whose ulp
//    is 2^24) yields u = ceil(T0 / 2^24) * 2^24 exactly; q = u - T0 is the
//    digit and u / 2^24 the carry, since T0 + q = u;
//  * R = 2^256 = 2^(10*24 + 16): ten 24-bit steps and a final 16-bit one
//    (same trick with 2^68, ulp 2^16); the result is (a*b + Q*p) / 2^256 <
//    a*b / 2^256 + p < 2p for a, b < 2p, then one conditional subtraction;
//  * normalisation uses a round-toward-zero add of 2^76 for floor(x / 2^24).
//
// Every constant is an exact power of two or a 24-bit digit of p; nothing
// depends on the rounding of an inexact operation.
#pragma once
#include "fr.cuh"

namespace pk {

namespace f64 {

constexpr double kTwo52 = 4503599627370496.0;            // 2^52
constexpr double kTwo68 = 295147905179352825856.0;       // 2^68
constexpr double kTwo76 = 75557863725914323419136.0;     // 2^76
constexpr double kInv24 = 1.0 / 16777216.0;              // 2^-24

// p in 24-bit digits, least significant first (digit 0 is 1).
__device__ __forceinline__ double pdig(int j) {
  constexpr double P[11] = {1.0,       16094192.0, 9520097.0,  7977328.0,
                            3401800.0, 5791016.0,  11960705.0, 12079173.0,
                            3252265.0, 5141217.0,  12388.0};
  return P[j];
}

// an integer v < 2^32 as a double: the bits 0x43300000:v are 2^52 + v.
__device__ __forceinline__ double dbl(uint32_t v) {
  return __hiloint2double(0x43300000, (int)v) - kTwo52;
}

// the 11 24-bit digits of a 256-bit value
__device__ __forceinline__ void digits(const Fr& b, double* B) {
  const uint32_t M = 0xFFFFFFu;
  B[0] = dbl(b.v[0] & M);
  B[1] = dbl(__funnelshift_r(b.v[0], b.v[1], 24) & M);
  B[2] = dbl(__funnelshift_r(b.v[1], b.v[2], 16) & M);
  B[3] = dbl(b.v[2] >> 8);
  B[4] = dbl(b.v[3] & M);
  B[5] = dbl(__funnelshift_r(b.v[3], b.v[4], 24) & M);
  B[6] = dbl(__funnelshift_r(b.v[4], b.v[5], 16) & M);
  B[7] = dbl(b.v[5] >> 8);
  B[8] = dbl(b.v[6] & M);
  B[9] = dbl(__funnelshift_r(b.v[6], b.v[7], 24) & M);
  B[10] = dbl(b.v[7] >> 16);
}

// One 24-bit Montgomery step on the column window T (T[0] complete): add
// q * p with q = -T[0] mod 2^24, carry T[0] / 2^24 into T[1], shift down.
__device__ __forceinline__ void step24(double* T) {
  const double u = __dadd_ru(T[0], kTwo76) - kTwo76;
  const double q = u - T[0];
  T[1] = fma(u, kInv24, T[1]);
#pragma unroll
  for (int j = 1; j < 11; j++) T[j] = fma(q, pdig(j), T[j]);
#pragma unroll
  for (int j = 0; j < 10; j++) T[j] = T[j + 1];
  T[10] = 0.0;
}

// The last 16-bit step, normalisation to 24-bit digits, and the shift by 16
// bits packed into eight 32-bit words; then one conditional subtraction.
__device__ __forceinline__ Fr tail16(double* T) {
  const double u = __dadd_ru(T[0], kTwo68) - kTwo68;
  const double q = u - T[0];
  T[0] = u;
#pragma unroll
  for (int j = 1; j < 11; j++) T[j] = fma(q, pdig(j), T[j]);
  uint32_t d[12];
  double x = T[0];
#pragma unroll
  for (int k = 0; k < 11; k++) {
    const double w = __dadd_rz(x, kTwo76) - kTwo76;
    d[k] = (uint32_t)__double2loint((x - w) + kTwo52);
    x = k < 10 ? fma(w, kInv24, T[k + 1]) : w * kInv24;
  }
  d[11] = (uint32_t)__double2loint(x + kTwo52);
  Fr r;
  r.v[0] = (d[0] >> 16) | (d[1] << 8);
  r.v[1] = d[2] | (d[3] << 24);
  r.v[2] = (d[3] >> 8) | (d[4] << 16);
  r.v[3] = (d[4] >> 16) | (d[5] << 8);
  r.v[4] = d[6] | (d[7] << 24);
  r.v[5] = (d[7] >> 8) | (d[8] << 16);
  r.v[6] = (d[8] >> 16) | (d[9] << 8);
  r.v[7] = d[10] | (d[11] << 24);
  return fr_reduce_once(r);
}

}  // namespace f64

// a * b * 2^-256 mod p for a, b < 2p; result < p (same value as fr_mul).
__device__ __forceinline__ Fr fr_mul_f64(const Fr& a, const Fr& b) {
  double A[11], B[11], T[11];
  f64::digits(a, A);
  f64::digits(b, B);
#pragma unroll
  for (int j = 0; j < 11; j++) T[j] = 0.0;
#pragma unroll
  for (int i = 0; i < 11; i++) {
#pragma unroll
    for (int j = 0; j < 11; j++) T[j] = fma(A[i], B[j], T[j]);
    if (i < 10) f64::step24(T);
  }
  return f64::tail16(T);
}

// fr_mul_f64 with the first operand already in digit form (A: the 11 digits
// f64::digits produced, e.g. a twiddle converted once and shared).
__device__ __forceinline__ Fr fr_mul_f64_digits(const double* A, const Fr& b) {
  double B[11], T[11];
  f64::digits(b, B);
#pragma unroll
  for (int j = 0; j < 11; j++) T[j] = 0.0;
#pragma unroll
  for (int i = 0; i < 11; i++) {
    const double ai = A[i];
#pragma unroll
    for (int j = 0; j < 11; j++) T[j] = fma(ai, B[j], T[j]);
    if (i < 10) f64::step24(T);
  }
  return f64::tail16(T);
}

// a^2 * 2^-256 mod p for a < 2p; result < p (same value as fr_sqr).  The 55
// cross products are taken once with a doubled operand (2 a_i < 2^25, so a
// product stays below 2^49 and a column below 2^53 as above).
__device__ __forceinline__ Fr fr_sqr_f64(const Fr& a) {
  double A[11], T[11];
  f64::digits(a, A);
#pragma unroll
  for (int j = 0; j < 11; j++) T[j] = 0.0;
#pragma unroll
  for (int i = 0; i < 11; i++) {
    T[i] = fma(A[i], A[i], T[i]);
    const double a2 = A[i] + A[i];
#pragma unroll
    for (int j = i + 1; j < 11; j++) T[j] = fma(a2, A[j], T[j]);
    if (i < 10) f64::step24(T);
  }
  return f64::tail16(T);
}

// a * 2^-256 mod p (Montgomery -> canonical) for any 256-bit a: the
// reduction steps alone, without a product; result < p.
__device__ __forceinline__ Fr fr_from_mont_f64(const Fr& a) {
  double T[11];
  f64::digits(a, T);
#pragma unroll
  for (int i = 0; i < 10; i++) f64::step24(T);
  return f64::tail16(T);
}

}  // namespace pk
