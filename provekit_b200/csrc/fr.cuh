// fr.cuh -- BN254 scalar field (Fr) arithmetic for sm_100a.
//
// An element is 8 x 32-bit little-endian limbs in registers; in memory it is
// the arkworks layout (4 x u64 LE == 8 x u32 LE), 32 bytes, 32-byte aligned.
// Multiplication is word-level CIOS Montgomery (Koc, Acar, Kaliski 1996) with
// R = 2^256, written as explicit PTX carry chains (mad.lo.cc / madc.hi.cc) so
// that every partial product is one IMAD-class instruction.  This replaces
// ark-ff's Fr multiply and bn254_multiplier::scalar_{mul,sqr}
// (skyscraper/bn254-multiplier/src/scalar.rs:12-132); outputs are fully
// reduced, as ark-ff stores them.
#pragma once
#include <cstdint>

namespace pk {

// p = 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001
#define PK_P0 0xf0000001u
#define PK_P1 0x43e1f593u
#define PK_P2 0x79b97091u
#define PK_P3 0x2833e848u
#define PK_P4 0x8181585du
#define PK_P5 0xb85045b6u
#define PK_P6 0xe131a029u
#define PK_P7 0x30644e72u
#define PK_MU 0xefffffffu  // -p^-1 mod 2^32

struct Fr {
  uint32_t v[8];
};

__device__ __forceinline__ Fr fr_zero() {
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = 0;
  return r;
}

// Montgomery form of 1 (2^256 mod p).
__device__ __forceinline__ Fr fr_one_mont() {
  Fr r;
  r.v[0] = 0x4ffffffbu; r.v[1] = 0xac96341cu; r.v[2] = 0x9f60cd29u; r.v[3] = 0x36fc7695u;
  r.v[4] = 0x7879462eu; r.v[5] = 0x666ea36fu; r.v[6] = 0x9a07df2fu; r.v[7] = 0x0e0a77c1u;
  return r;
}

__device__ __forceinline__ Fr fr_load(const uint64_t* base, size_t idx) {
  const uint4* p = reinterpret_cast<const uint4*>(base + 4 * idx);
  uint4 a = p[0], b = p[1];
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}

__device__ __forceinline__ Fr fr_load_ro(const uint64_t* base, size_t idx) {
  const uint4* p = reinterpret_cast<const uint4*>(base + 4 * idx);
  uint4 a = __ldg(p), b = __ldg(p + 1);
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}

__device__ __forceinline__ void fr_store(uint64_t* base, size_t idx, const Fr& x) {
  uint4* p = reinterpret_cast<uint4*>(base + 4 * idx);
  p[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  p[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// x - p if x >= p (x < 2^256).
__device__ __forceinline__ Fr fr_reduce_once(const Fr& x) {
  Fr d;
  uint32_t borrow;
  asm("sub.cc.u32  %0, %9,  %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d.v[0]), "=r"(d.v[1]), "=r"(d.v[2]), "=r"(d.v[3]), "=r"(d.v[4]), "=r"(d.v[5]),
        "=r"(d.v[6]), "=r"(d.v[7]), "=r"(borrow)
      : "r"(x.v[0]), "r"(x.v[1]), "r"(x.v[2]), "r"(x.v[3]), "r"(x.v[4]), "r"(x.v[5]),
        "r"(x.v[6]), "r"(x.v[7]), "n"(PK_P0), "n"(PK_P1), "n"(PK_P2), "n"(PK_P3), "n"(PK_P4),
        "n"(PK_P5), "n"(PK_P6), "n"(PK_P7));
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = borrow ? x.v[i] : d.v[i];
  return r;
}

// (a + b) mod p for a, b < p.
__device__ __forceinline__ Fr fr_add(const Fr& a, const Fr& b) {
  Fr s;
  asm("add.cc.u32  %0, %8,  %16;\n\t"
      "addc.cc.u32 %1, %9,  %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(s.v[0]), "=r"(s.v[1]), "=r"(s.v[2]), "=r"(s.v[3]), "=r"(s.v[4]), "=r"(s.v[5]),
        "=r"(s.v[6]), "=r"(s.v[7])
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]),
        "r"(a.v[6]), "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]),
        "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  return fr_reduce_once(s);
}

// (a - b) mod p for a, b < p.
__device__ __forceinline__ Fr fr_sub(const Fr& a, const Fr& b) {
  Fr d;
  uint32_t borrow;
  asm("sub.cc.u32  %0, %9,  %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d.v[0]), "=r"(d.v[1]), "=r"(d.v[2]), "=r"(d.v[3]), "=r"(d.v[4]), "=r"(d.v[5]),
        "=r"(d.v[6]), "=r"(d.v[7]), "=r"(borrow)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]),
        "r"(a.v[6]), "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]),
        "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  // add p & borrow-mask
  Fr r;
  asm("add.cc.u32  %0, %8,  %16;\n\t"
      "addc.cc.u32 %1, %9,  %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
        "=r"(r.v[6]), "=r"(r.v[7])
      : "r"(d.v[0]), "r"(d.v[1]), "r"(d.v[2]), "r"(d.v[3]), "r"(d.v[4]), "r"(d.v[5]),
        "r"(d.v[6]), "r"(d.v[7]), "r"(PK_P0 & borrow), "r"(PK_P1 & borrow), "r"(PK_P2 & borrow),
        "r"(PK_P3 & borrow), "r"(PK_P4 & borrow), "r"(PK_P5 & borrow), "r"(PK_P6 & borrow),
        "r"(PK_P7 & borrow));
  return r;
}

// t[0..8] += a * b  (two carry chains: low halves into t0..t7 with the
// carry into t8, high halves into t1..t8).  Requires the sum < 2^288.
#define PK_ROW(T, A, B)                                                                          \
  asm("mad.lo.cc.u32  %0, %9,  %17, %0;\n\t"                                                    \
      "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"                                                    \
      "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"                                                    \
      "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"                                                    \
      "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"                                                    \
      "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"                                                    \
      "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"                                                    \
      "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"                                                    \
      "addc.u32       %8, %8, 0;"                                                                \
      : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),      \
        "+r"(T[7]), "+r"(T[8])                                                                   \
      : "r"(A[0]), "r"(A[1]), "r"(A[2]), "r"(A[3]), "r"(A[4]), "r"(A[5]), "r"(A[6]), "r"(A[7]),  \
        "r"(B));                                                                                 \
  asm("mad.hi.cc.u32  %0, %8,  %16, %0;\n\t"                                                    \
      "madc.hi.cc.u32 %1, %9,  %16, %1;\n\t"                                                    \
      "madc.hi.cc.u32 %2, %10, %16, %2;\n\t"                                                    \
      "madc.hi.cc.u32 %3, %11, %16, %3;\n\t"                                                    \
      "madc.hi.cc.u32 %4, %12, %16, %4;\n\t"                                                    \
      "madc.hi.cc.u32 %5, %13, %16, %5;\n\t"                                                    \
      "madc.hi.cc.u32 %6, %14, %16, %6;\n\t"                                                    \
      "madc.hi.u32    %7, %15, %16, %7;"                                                         \
      : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]),      \
        "+r"(T[8])                                                                               \
      : "r"(A[0]), "r"(A[1]), "r"(A[2]), "r"(A[3]), "r"(A[4]), "r"(A[5]), "r"(A[6]), "r"(A[7]),  \
        "r"(B))

// t[0..8] += m * p, as PK_ROW with the modulus as immediates.
#define PK_ROW_P(T, M)                                                                           \
  asm("mad.lo.cc.u32  %0, %9,  %10, %0;\n\t"                                                    \
      "madc.lo.cc.u32 %1, %9,  %11, %1;\n\t"                                                    \
      "madc.lo.cc.u32 %2, %9,  %12, %2;\n\t"                                                    \
      "madc.lo.cc.u32 %3, %9,  %13, %3;\n\t"                                                    \
      "madc.lo.cc.u32 %4, %9,  %14, %4;\n\t"                                                    \
      "madc.lo.cc.u32 %5, %9,  %15, %5;\n\t"                                                    \
      "madc.lo.cc.u32 %6, %9,  %16, %6;\n\t"                                                    \
      "madc.lo.cc.u32 %7, %9,  %17, %7;\n\t"                                                    \
      "addc.u32       %8, %8, 0;"                                                                \
      : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),      \
        "+r"(T[7]), "+r"(T[8])                                                                   \
      : "r"(M), "n"(PK_P0), "n"(PK_P1), "n"(PK_P2), "n"(PK_P3), "n"(PK_P4), "n"(PK_P5),          \
        "n"(PK_P6), "n"(PK_P7));                                                                 \
  asm("mad.hi.cc.u32  %0, %8,  %9,  %0;\n\t"                                                    \
      "madc.hi.cc.u32 %1, %8,  %10, %1;\n\t"                                                    \
      "madc.hi.cc.u32 %2, %8,  %11, %2;\n\t"                                                    \
      "madc.hi.cc.u32 %3, %8,  %12, %3;\n\t"                                                    \
      "madc.hi.cc.u32 %4, %8,  %13, %4;\n\t"                                                    \
      "madc.hi.cc.u32 %5, %8,  %14, %5;\n\t"                                                    \
      "madc.hi.cc.u32 %6, %8,  %15, %6;\n\t"                                                    \
      "madc.hi.u32    %7, %8,  %16, %7;"                                                         \
      : "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]),      \
        "+r"(T[8])                                                                               \
      : "r"(M), "n"(PK_P0), "n"(PK_P1), "n"(PK_P2), "n"(PK_P3), "n"(PK_P4), "n"(PK_P5),          \
        "n"(PK_P6), "n"(PK_P7))

// Montgomery product a * b * 2^-256 mod p.  Inputs a, b < 2p; the CIOS
// accumulator then stays below 3p at every word boundary and below 2^288
// inside a word step, so 9 limbs suffice.  Output fully reduced (< p) when
// a, b < p (one conditional subtraction; t < 2p), and < p after two
// conditional subtractions for a, b < 2p (t < 3p).
template <bool kTwoSub = false>
__device__ __forceinline__ Fr fr_mul(const Fr& a, const Fr& b) {
  uint32_t t[9];
#pragma unroll
  for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    PK_ROW(t, a.v, b.v[i]);
    uint32_t m = t[0] * PK_MU;
    PK_ROW_P(t, m);
    // t[0] is now 0: shift one word down.
#pragma unroll
    for (int j = 0; j < 8; j++) t[j] = t[j + 1];
    t[8] = 0;
  }
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = t[i];
  r = fr_reduce_once(r);
  if (kTwoSub) r = fr_reduce_once(r);
  return r;
}

// Montgomery square a^2 * 2^-256 mod p for a < p, as separated operand
// scanning (SOS): the 28 cross products a_i a_j (i < j) once, doubled, plus
// the 8 diagonal squares -- 36 word products instead of 64 -- then the
// word-by-word Montgomery reduction.  Accumulation uses 64-bit
// multiply-adds; the result is fully reduced.
__device__ __forceinline__ Fr fr_sqr(const Fr& a) {
  const uint32_t P[8] = {PK_P0, PK_P1, PK_P2, PK_P3, PK_P4, PK_P5, PK_P6, PK_P7};
  uint32_t t[17];
#pragma unroll
  for (int i = 0; i < 17; i++) t[i] = 0;
#pragma unroll
  for (int i = 0; i < 7; i++) {
    uint64_t c = 0;
#pragma unroll
    for (int j = i + 1; j < 8; j++) {
      uint64_t s = (uint64_t)a.v[i] * a.v[j] + t[i + j] + c;
      t[i + j] = (uint32_t)s;
      c = s >> 32;
    }
    t[i + 8] = (uint32_t)c;
  }
#pragma unroll
  for (int k = 15; k > 0; k--) t[k] = (t[k] << 1) | (t[k - 1] >> 31);
  t[0] <<= 1;
  uint64_t c = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    uint64_t sq = (uint64_t)a.v[i] * a.v[i];
    uint64_t s = (uint64_t)t[2 * i] + (uint32_t)sq + c;
    t[2 * i] = (uint32_t)s;
    c = s >> 32;
    s = (uint64_t)t[2 * i + 1] + (uint32_t)(sq >> 32) + c;
    t[2 * i + 1] = (uint32_t)s;
    c = s >> 32;
  }
  // reduction: t += m_i * p * 2^(32 i), i = 0..7 (a^2 < p^2 keeps t < 2^512 + p 2^256)
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t m = t[i] * PK_MU;
    uint64_t c2 = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      uint64_t s = (uint64_t)m * P[j] + t[i + j] + c2;
      t[i + j] = (uint32_t)s;
      c2 = s >> 32;
    }
#pragma unroll
    for (int k = i + 8; k < 17; k++) {
      uint64_t s = (uint64_t)t[k] + c2;
      t[k] = (uint32_t)s;
      c2 = s >> 32;
    }
  }
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = t[i + 8];
  return fr_reduce_once(r);
}

// canonical -> Montgomery: a * R^2 * R^-1
__device__ __forceinline__ Fr fr_to_mont(const Fr& a) {
  Fr r2;
  r2.v[0] = 0xae216da7u; r2.v[1] = 0x1bb8e645u; r2.v[2] = 0xe35c59e3u; r2.v[3] = 0x53fe3ab1u;
  r2.v[4] = 0x53bb8085u; r2.v[5] = 0x8c49833du; r2.v[6] = 0x7f4e44a5u; r2.v[7] = 0x0216d0b1u;
  return fr_mul(a, r2);
}

// Montgomery -> canonical: a * 1 * R^-1
// Montgomery -> canonical, a * 2^-256 mod p, for any 256-bit a: the
// word-by-word Montgomery reduction alone (REDC, 8 x (1 + 16) multiply-adds
// on the integer pipe, no product); t < 2^256 + p 2^256 keeps 9 words, the
// result is < p + 1 before the one conditional subtraction.
__device__ __forceinline__ Fr fr_from_mont(const Fr& a) {
  uint32_t t[9];
#pragma unroll
  for (int i = 0; i < 8; i++) t[i] = a.v[i];
  t[8] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t m = t[0] * PK_MU;
    PK_ROW_P(t, m);
#pragma unroll
    for (int j = 0; j < 8; j++) t[j] = t[j + 1];
    t[8] = 0;
  }
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = t[i];
  return fr_reduce_once(r);
}

__device__ __forceinline__ bool fr_eq(const Fr& a, const Fr& b) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) d |= a.v[i] ^ b.v[i];
  return d == 0;
}

}  // namespace pk
