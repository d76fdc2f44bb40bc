// sky_host.hpp -- host-side Skyscraper permutation (skyscraper/core/src/
// reference.rs:49-98) on canonical values, for the Fiat-Shamir transcript.
// ss: r += l^2 * 2^-256 + RC (the Montgomery square of a canonical value);
// bb: r += bar(l) + RC.
#pragma once
#include <cstdint>
#include <cstring>

#include "fr_host.hpp"

namespace pk {

struct HostSky {
  static const uint64_t* rc(int k) {
    static const uint64_t RC[18][4] = {
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
    return RC[k];
  }
  // sbox (bar.rs:40-42) on the 8 bytes of a word at once: rotations within
  // each byte, rotl_k(v) = ((v & high k bits) >> (8 - k)) | ((v & low bits) << k)
  static uint64_t sbox8(uint64_t v) {
    const uint64_t nv = ~v;
    const uint64_t r1 = ((nv & 0x8080808080808080ULL) >> 7) | ((nv & 0x7f7f7f7f7f7f7f7fULL) << 1);
    const uint64_t r2 = ((v & 0xc0c0c0c0c0c0c0c0ULL) >> 6) | ((v & 0x3f3f3f3f3f3f3f3fULL) << 2);
    const uint64_t r3 = ((v & 0xe0e0e0e0e0e0e0e0ULL) >> 5) | ((v & 0x1f1f1f1f1f1f1f1fULL) << 3);
    const uint64_t t = v ^ (r1 & r2 & r3);
    return ((t & 0x8080808080808080ULL) >> 7) | ((t & 0x7f7f7f7f7f7f7f7fULL) << 1);
  }
  // any 256-bit value -> [0, p)
  static HostFr reduce(HostFr x) {
    while (!x.is_canonical()) x = HostFr::sub_p(x);
    return x;
  }
  static HostFr bar(const HostFr& x) {
    HostFr y;
    y.l[0] = sbox8(x.l[2]);
    y.l[1] = sbox8(x.l[3]);
    y.l[2] = sbox8(x.l[0]);
    y.l[3] = sbox8(x.l[1]);
    return reduce(y);
  }
  static void round(int k, bool is_bar, HostFr& l, HostFr& r) {
    HostFr f = is_bar ? bar(l) : HostFr::mul(l, l);
    HostFr nl = HostFr::add(HostFr::add(r, f), HostFr::from_limbs(rc(k)));
    r = l;
    l = nl;
  }
  // reference::permute (reference.rs:49-60) on canonical (l, r)
  static void permute(HostFr& l, HostFr& r) {
    for (int k = 0; k < 18; k++) round(k, k == 6 || k == 7 || k == 10 || k == 11, l, r);
  }
  // reference::compress (reference.rs:41-46): permute(l, r).0 + l, canonical
  static HostFr compress(const HostFr& l, const HostFr& r) {
    HostFr a = l, b = r;
    permute(a, b);
    return HostFr::add(a, l);
  }
};

}  // namespace pk
