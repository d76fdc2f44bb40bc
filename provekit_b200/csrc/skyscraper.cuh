// skyscraper.cuh -- Skyscraper v2 two-to-one compression over BN254 Fr on the
// device (skyscraper/core/src/generic.rs:77-102, reference.rs:41-98).
//
// Inputs and outputs are canonical little-endian limbs (not Montgomery).
// Every intermediate value is kept fully reduced in [0, p): the reference's
// partial-reduction bookkeeping (reduce.rs:15-55) only chooses representatives,
// and bar() reduces its input first (bar.rs:15-31), so the output bytes depend
// only on values mod p.  The square is the Montgomery square x^2 * 2^-256
// (the reference's scalar_sqr, equal to l.square() * SIGMA_INV in
// reference.rs:64).
#pragma once
#include "fr.cuh"
#include "fr_f64.cuh"

namespace pk {

// Skyscraper round constants (skyscraper/core/src/constants.rs:30-49) as
// 8 x u32 LE limbs; RC[0] = RC[17] = 0.
__constant__ uint32_t kSkyRC[18][8] = {
    {0, 0, 0, 0, 0, 0, 0, 0},
    {0x270bd744u, 0x903c4324u, 0x08a7d269u, 0x873125f7u, 0x06c83855u, 0x081dd279u, 0xea6d7667u, 0x276b1823u},
    {0x4b378d71u, 0x7ac8edbbu, 0xd99e2cb7u, 0xe29d79f3u, 0x4c1a5a18u, 0x75141791u, 0x58a484a6u, 0x0cf02bd7u},
    {0x69e5bc36u, 0xfa7adc67u, 0x7cca387du, 0x1c3f8e29u, 0x63481db0u, 0x0eb7730du, 0x18ede544u, 0x25b0e03fu},
    {0x2f03cfb7u, 0x57847e65u, 0x68873404u, 0x33440b96u, 0x49af80bcu, 0x955a32e8u, 0xbe14ae70u, 0x002882fcu},
    {0x6257d4d7u, 0x97923139u, 0x1b37d3c1u, 0x29989c3eu, 0x7f1277bau, 0x12ef02b4u, 0x1e2b7a9cu, 0x039ad857u},
    {0xabbb7887u, 0xb5b48465u, 0xe6ba2d2bu, 0xa72a6bc5u, 0x712f7b29u, 0x4cd48043u, 0x0fc1fc1au, 0x1142d541u},
    {0x059075d3u, 0x7ab2c156u, 0x047999b2u, 0x17cb3594u, 0x98f289f7u, 0x44f2c935u, 0x69bc0becu, 0x1d78439fu},
    {0x138b8edbu, 0x05d7a965u, 0xd55c48b1u, 0x36ef35a3u, 0xac6f1628u, 0x8ddfb8a1u, 0x08f4ff82u, 0x258588a5u},
    {0xfccb49e9u, 0x1596fb9au, 0x9a09a95bu, 0x9a7367d6u, 0x84e4c157u, 0x9bc43f69u, 0xd2f514feu, 0x13087879u},
    {0x3b4109fau, 0x295ccd23u, 0xed868012u, 0xe1d72f89u, 0x4bc88a8eu, 0x2e9e1eeau, 0x98c45232u, 0x17dadee8u},
    {0xaa1f486fu, 0x9a8590b4u, 0x30e9130eu, 0xb75834b4u, 0x34d5de31u, 0xb8e90b10u, 0x46e7f4a6u, 0x295c6d15u},
    {0x4c6eb892u, 0x850adcb7u, 0x05b92fc3u, 0x07699ef3u, 0xa1720f2du, 0x4ef96a2bu, 0x1d3ed446u, 0x1288ca0eu},
    {0x49d1b5eeu, 0x01960f93u, 0x69371c69u, 0x8ccad307u, 0x91c98662u, 0xe5c81e89u, 0x1ae023f3u, 0x17563b4du},
    {0x76b32917u, 0x6ba01e94u, 0xdd977bc9u, 0xa1cb0a3au, 0x5815f030u, 0x86815a94u, 0xe91a1eeau, 0x2869043bu},
    {0x5511d976u, 0x81776c88u, 0x47f414e7u, 0x7475d34fu, 0x095d96cfu, 0x5d090056u, 0xff59e79au, 0x14941f0au},
    {0x8fc8c034u, 0xbc40b4fdu, 0xcce4fd48u, 0xbb7142c3u, 0x8a39005au, 0x31835675u, 0x90f4379fu, 0x1ce337a1u},
    {0, 0, 0, 0, 0, 0, 0, 0},
};

// k * p for k = 0..5 (skyscraper/core/src/constants.rs:8-15), u32 limbs.
__constant__ uint32_t kModMul[6][8] = {
    {0, 0, 0, 0, 0, 0, 0, 0},
    {0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u, 0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u},
    {0xe0000002u, 0x87c3eb27u, 0xf372e122u, 0x5067d090u, 0x0302b0bau, 0x70a08b6du, 0xc2634053u, 0x60c89ce5u},
    {0xd0000003u, 0xcba5e0bbu, 0x6d2c51b3u, 0x789bb8d9u, 0x84840917u, 0x28f0d123u, 0xa394e07du, 0x912ceb58u},
    {0xc0000004u, 0x0f87d64fu, 0xe6e5c245u, 0xa0cfa121u, 0x06056174u, 0xe14116dau, 0x84c680a6u, 0xc19139cbu},
    {0xb0000005u, 0x5369cbe3u, 0x609f32d6u, 0xc903896au, 0x8786b9d1u, 0x99915c90u, 0x65f820d0u, 0xf1f5883eu},
};

// Full reduction of any 256-bit value: subtract q*p with q = top limb /
// (p_top + 1) <= floor(x / p), leaving x < 2p, then one conditional subtract.
__device__ __forceinline__ Fr sky_reduce_any(const Fr& x) {
  uint32_t q = x.v[7] / (PK_P7 + 1u);
  Fr m;
#pragma unroll
  for (int i = 0; i < 8; i++) m.v[i] = kModMul[q][i];
  Fr d;
  asm("sub.cc.u32  %0, %8,  %16;\n\t"
      "subc.cc.u32 %1, %9,  %17;\n\t"
      "subc.cc.u32 %2, %10, %18;\n\t"
      "subc.cc.u32 %3, %11, %19;\n\t"
      "subc.cc.u32 %4, %12, %20;\n\t"
      "subc.cc.u32 %5, %13, %21;\n\t"
      "subc.cc.u32 %6, %14, %22;\n\t"
      "subc.u32    %7, %15, %23;"
      : "=r"(d.v[0]), "=r"(d.v[1]), "=r"(d.v[2]), "=r"(d.v[3]), "=r"(d.v[4]), "=r"(d.v[5]),
        "=r"(d.v[6]), "=r"(d.v[7])
      : "r"(x.v[0]), "r"(x.v[1]), "r"(x.v[2]), "r"(x.v[3]), "r"(x.v[4]), "r"(x.v[5]),
        "r"(x.v[6]), "r"(x.v[7]), "r"(m.v[0]), "r"(m.v[1]), "r"(m.v[2]), "r"(m.v[3]),
        "r"(m.v[4]), "r"(m.v[5]), "r"(m.v[6]), "r"(m.v[7]));
  return fr_reduce_once(d);
}

// Per-byte sbox (bar.rs:40-42) on the 4 bytes of a word:
// sbox(v) = rotl1(v ^ (rotl1(~v) & rotl2(v) & rotl3(v))), rotations within bytes.
__device__ __forceinline__ uint32_t sky_sbox4(uint32_t v) {
  uint32_t nv = ~v;
  uint32_t r1 = ((nv & 0x80808080u) >> 7) | ((nv & 0x7f7f7f7fu) << 1);
  uint32_t r2 = ((v & 0xc0c0c0c0u) >> 6) | ((v & 0x3f3f3f3fu) << 2);
  uint32_t r3 = ((v & 0xe0e0e0e0u) >> 5) | ((v & 0x1f1f1f1fu) << 3);
  uint32_t t = v ^ (r1 & r2 & r3);
  return ((t & 0x80808080u) >> 7) | ((t & 0x7f7f7f7fu) << 1);
}

// bar (bar.rs:15-31) on a canonical value: swap the 16-byte halves, sbox
// every byte, reduce.
__device__ __forceinline__ Fr sky_bar(const Fr& x) {
  Fr y;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    y.v[i] = sky_sbox4(x.v[i + 4]);
    y.v[i + 4] = sky_sbox4(x.v[i]);
  }
  return sky_reduce_any(y);
}

__device__ __forceinline__ Fr sky_rc(int k) {
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = kSkyRC[k][i];
  return r;
}

// Skyscraper v2 compress(l, r) for arbitrary 256-bit inputs.  Rounds 6, 7,
// 10 and 11 use bar, the others the Montgomery square; RC[0] = RC[17] = 0.
// The round loop is kept rolled: one compression is ~5k instructions and
// unrolling it only costs registers (occupancy) at every call site.
__device__ __forceinline__ Fr sky_compress(Fr l, Fr r) {
  l = sky_reduce_any(l);
  r = sky_reduce_any(r);
  const Fr t = l;
#pragma unroll 1
  for (int k = 0; k < 18; k++) {
    const bool is_bar = (k == 6 || k == 7 || k == 10 || k == 11);
    Fr f = is_bar ? sky_bar(l) : fr_sqr_f64(l);
    Fr nl = fr_add(r, f);
    nl = fr_add(nl, sky_rc(k));
    r = l;
    l = nl;
  }
  return fr_add(l, t);
}

}  // namespace pk
