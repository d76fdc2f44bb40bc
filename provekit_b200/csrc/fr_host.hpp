// fr_host.hpp -- host-side BN254 Fr for the few scalar computations the
// library does on the CPU between kernels (sampler conversion, twiddle seeds,
// n^-1, sumcheck round-polynomial bookkeeping).  4 x u64 limbs, Montgomery
// form R = 2^256, fully reduced (ark-ff semantics); CIOS multiplication.
#pragma once
#include <cstdint>
#include <cstring>

namespace pk {

struct HostFr {
  uint64_t l[4] = {0, 0, 0, 0};

  static constexpr uint64_t P[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                                    0xb85045b68181585dULL, 0x30644e72e131a029ULL};
  static constexpr uint64_t INV = 0xc2e1f593efffffffULL;
  static constexpr uint64_t R2[4] = {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL,
                                     0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL};

  static HostFr from_limbs(const uint64_t* p) {
    HostFr r;
    memcpy(r.l, p, 32);
    return r;
  }
  static HostFr one() {  // Montgomery 1
    HostFr r;
    r.l[0] = 0xac96341c4ffffffbULL; r.l[1] = 0x36fc76959f60cd29ULL;
    r.l[2] = 0x666ea36f7879462eULL; r.l[3] = 0x0e0a77c19a07df2fULL;
    return r;
  }
  static HostFr zero() { return HostFr(); }

  bool is_canonical() const {
    for (int i = 3; i >= 0; i--) {
      if (l[i] != P[i]) return l[i] < P[i];
    }
    return false;
  }
  bool operator==(const HostFr& o) const { return memcmp(l, o.l, 32) == 0; }

  static HostFr mul(const HostFr& a, const HostFr& b) {
    typedef unsigned __int128 u128;
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
      u128 c = 0;
      for (int j = 0; j < 4; j++) {
        c += (u128)a.l[j] * b.l[i] + t[j];
        t[j] = (uint64_t)c;
        c >>= 64;
      }
      c += t[4];
      t[4] = (uint64_t)c;
      t[5] = (uint64_t)(c >> 64);
      uint64_t m = t[0] * INV;
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
    HostFr r;
    memcpy(r.l, t, 32);
    while (t[4] != 0 || !r.is_canonical()) {
      uint64_t borrow = 0;
      for (int i = 0; i < 4; i++) {
        u128 d = (u128)r.l[i] - P[i] - borrow;
        r.l[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) ? 1 : 0;
      }
      t[4] -= borrow;
    }
    return r;
  }
  static HostFr add(const HostFr& a, const HostFr& b) {
    typedef unsigned __int128 u128;
    HostFr r;
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
      c += (u128)a.l[i] + b.l[i];
      r.l[i] = (uint64_t)c;
      c >>= 64;
    }
    if (!r.is_canonical()) r = sub_p(r);
    return r;
  }
  static HostFr sub(const HostFr& a, const HostFr& b) {
    typedef unsigned __int128 u128;
    HostFr r;
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
      u128 d = (u128)a.l[i] - b.l[i] - borrow;
      r.l[i] = (uint64_t)d;
      borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    if (borrow) {
      u128 c = 0;
      for (int i = 0; i < 4; i++) {
        c += (u128)r.l[i] + P[i];
        r.l[i] = (uint64_t)c;
        c >>= 64;
      }
    }
    return r;
  }
  static HostFr sub_p(const HostFr& a) {
    typedef unsigned __int128 u128;
    HostFr r;
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
      u128 d = (u128)a.l[i] - P[i] - borrow;
      r.l[i] = (uint64_t)d;
      borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return r;
  }
  static HostFr to_mont(const HostFr& a) {
    HostFr r2;
    memcpy(r2.l, R2, 32);
    return mul(a, r2);
  }
  static HostFr from_mont(const HostFr& a) {
    HostFr one_c;
    one_c.l[0] = 1;
    return mul(a, one_c);
  }
  static HostFr from_u64(uint64_t v) {
    HostFr c;
    c.l[0] = v;
    return to_mont(c);
  }
  static HostFr pow(const HostFr& base, const uint64_t e[4]) {
    HostFr acc = one(), b = base;
    for (int i = 0; i < 256; i++) {
      if ((e[i / 64] >> (i % 64)) & 1) acc = mul(acc, b);
      b = mul(b, b);
    }
    return acc;
  }
  static HostFr pow_u64(const HostFr& base, uint64_t e) {
    HostFr acc = one(), b = base;
    for (; e; e >>= 1) {
      if (e & 1) acc = mul(acc, b);
      b = mul(b, b);
    }
    return acc;
  }
  static HostFr inv(const HostFr& a) {
    uint64_t e[4] = {P[0] - 2, P[1], P[2], P[3]};
    return pow(a, e);
  }
  // Fr::get_root_of_unity(n), n = 2^k <= 2^28: GENERATOR = 5 raised to
  // (p-1)/2^28, squared 28-k times (ark-ff's derivation for ark-bn254).
  static HostFr root_of_unity(uint64_t n) {
    int k = 0;
    while ((uint64_t(1) << k) < n) k++;
    // the 2^28-th root, exponentiated once per process (~400 products)
    static const HostFr w28 = [] {
      uint64_t t[4] = {P[0] - 1, P[1], P[2], P[3]};
      for (int i = 0; i < 28; i++) {
        t[0] = (t[0] >> 1) | (t[1] << 63);
        t[1] = (t[1] >> 1) | (t[2] << 63);
        t[2] = (t[2] >> 1) | (t[3] << 63);
        t[3] >>= 1;
      }
      return pow(from_u64(5), t);
    }();
    HostFr w = w28;
    for (int i = k; i < 28; i++) w = mul(w, w);
    return w;
  }
};

}  // namespace pk
