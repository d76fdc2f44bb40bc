// sumcheck_device.cuh -- device-side pieces of the Spartan zk-sumcheck used by
// the batched form: the transcript stand-in (same definition as the host's
// pkg_transcript_*), compute_blinding_coefficients_for_round
// (provekit/prover/src/whir_r1cs.rs:427-492) and the cubic evaluation
// (provekit/common/src/utils/sumcheck.rs:156-158), one thread per job.
#pragma once
#include "fr.cuh"
#include "skyscraper.cuh"

namespace pk {

// reference::permute (skyscraper/core/src/reference.rs:49-60) on canonical
// values: 18 rounds, square (Montgomery square of a canonical value = l^2 *
// SIGMA_INV) or bar, plus the round constant.
__device__ __forceinline__ void sky_permute(Fr& l, Fr& r) {
#pragma unroll 1
  for (int k = 0; k < 18; k++) {
    const bool is_bar = (k == 6 || k == 7 || k == 10 || k == 11);
    Fr f = is_bar ? sky_bar(l) : fr_sqr_f64(l);
    Fr nl = fr_add(fr_add(r, f), sky_rc(k));
    r = l;
    l = nl;
  }
}

struct DevTranscript {
  Fr l, r;  // canonical
  __device__ void init(const Fr& domain_canonical) {
    l = domain_canonical;
    r = fr_zero();
    sky_permute(l, r);
  }
  __device__ void absorb(const Fr& x_mont) {
    l = fr_add(l, fr_from_mont(x_mont));
    sky_permute(l, r);
  }
  __device__ Fr squeeze() {
    sky_permute(l, r);
    return fr_to_mont(l);
  }
};

__device__ __forceinline__ Fr dev_cubic(const Fr* c, const Fr& x) {
  Fr acc = fr_mul_f64(x, c[3]);
  acc = fr_mul_f64(fr_add(acc, c[2]), x);
  acc = fr_mul_f64(fr_add(acc, c[1]), x);
  return fr_add(acc, c[0]);
}

// (p + 1) / 2 in Montgomery form = 2^-1
__device__ __forceinline__ Fr fr_half_mont() {
  Fr one = fr_one_mont();
  // 2^-1 * R = (R + p) / 2 when R is odd... compute as one * half via shift:
  // R mod p is odd here, so (R mod p + p) / 2 is exact.
  Fr s;
  uint32_t carry = 0;
  // s = one + p (257 bits at most), then >> 1
  asm("add.cc.u32  %0, %9,  %17;\n\t"
      "addc.cc.u32 %1, %10, %18;\n\t"
      "addc.cc.u32 %2, %11, %19;\n\t"
      "addc.cc.u32 %3, %12, %20;\n\t"
      "addc.cc.u32 %4, %13, %21;\n\t"
      "addc.cc.u32 %5, %14, %22;\n\t"
      "addc.cc.u32 %6, %15, %23;\n\t"
      "addc.cc.u32 %7, %16, %24;\n\t"
      "addc.u32    %8, 0, 0;"
      : "=r"(s.v[0]), "=r"(s.v[1]), "=r"(s.v[2]), "=r"(s.v[3]), "=r"(s.v[4]), "=r"(s.v[5]),
        "=r"(s.v[6]), "=r"(s.v[7]), "=r"(carry)
      : "r"(one.v[0]), "r"(one.v[1]), "r"(one.v[2]), "r"(one.v[3]), "r"(one.v[4]), "r"(one.v[5]),
        "r"(one.v[6]), "r"(one.v[7]), "n"(PK_P0), "n"(PK_P1), "n"(PK_P2), "n"(PK_P3), "n"(PK_P4),
        "n"(PK_P5), "n"(PK_P6), "n"(PK_P7));
  Fr h;
#pragma unroll
  for (int i = 0; i < 7; i++) h.v[i] = (s.v[i] >> 1) | (s.v[i + 1] << 31);
  h.v[7] = (s.v[7] >> 1) | (carry << 31);
  return h;
}

// compute_blinding_coefficients_for_round (whir_r1cs.rs:427-492); g: n x 4,
// alphas: at least compute_for entries.
__device__ __forceinline__ void dev_blinding_coeffs(const Fr* g, int n, int compute_for,
                                                    const Fr* alphas, Fr out[4]) {
  bool all_fixed = false;
  int cf = compute_for;
  if (cf == n) {
    all_fixed = true;
    cf = n - 1;
  }
  Fr prefix = fr_zero(), suffix = fr_zero();
  for (int i = 0; i < cf; i++) prefix = fr_add(prefix, dev_cubic(g + 4 * i, alphas[i]));
  for (int i = cf + 1; i < n; i++)
    suffix = fr_add(suffix, fr_add(dev_cubic(g + 4 * i, fr_zero()), dev_cubic(g + 4 * i, fr_one_mont())));
  Fr pm = fr_one_mont();
  for (int i = 0; i < n - 1 - cf; i++) pm = fr_add(pm, pm);
  Fr sm = fr_mul_f64(pm, fr_half_mont());
  Fr cst = fr_add(fr_mul_f64(pm, prefix), fr_mul_f64(sm, suffix));
  const Fr* cur = g + 4 * cf;
  Fr res[4] = {fr_add(fr_mul_f64(pm, cur[0]), cst), fr_mul_f64(pm, cur[1]), fr_mul_f64(pm, cur[2]),
               fr_mul_f64(pm, cur[3])};
  if (all_fixed) {
    out[0] = dev_cubic(res, alphas[cf]);
    out[1] = out[2] = out[3] = fr_zero();
    return;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) out[k] = res[k];
}

// The Spartan round code below multiplies 14 times per pair; inlining every
// FP64 product makes a ~100 KB kernel that runs from cold instruction cache
// (small rounds took ~40 us whatever their size).  One out-of-line product
// keeps the kernel small.
static __device__ __noinline__ Fr fr_mul_call(const Fr a, const Fr b) { return fr_mul_f64(a, b); }

// One pair (t[j], t[j + q]) of a table; with kFold the live size is 4q and
// the top variable is folded first, t[j] += f (t[j+2q] - t[j]) and
// t[j+q] += f (t[j+3q] - t[j+q]), in place.
template <bool kFold>
__device__ __forceinline__ void round_pair(uint64_t* t, size_t j, size_t q, const Fr& fold, Fr& x0,
                                           Fr& x1) {
  x0 = fr_load(t, j);
  x1 = fr_load(t, j + q);
  if (kFold) {
    x0 = fr_add(x0, fr_mul_call(fold, fr_sub(fr_load(t, j + 2 * q), x0)));
    x1 = fr_add(x1, fr_mul_call(fold, fr_sub(fr_load(t, j + 3 * q), x1)));
    fr_store(t, j, x0);
    fr_store(t, j + q, x1);
  }
}

// The Spartan closure (whir_r1cs.rs:552-558) on one pair of each table,
// streaming the tables a, b, c, eq in turn so that only partial products
// stay live:
//   f(0)   = eq0 (a0 b0 - c0)
//   f(-1)  = (2eq0 - eq1) ((2a0 - a1)(2b0 - b1) - (2c0 - c1))
//   f(inf) = (eq1 - eq0)(a1 - a0)(b1 - b0)
template <bool kFold>
__device__ __forceinline__ void spartan_pair(uint64_t* const (&tabs)[4], size_t j, size_t q,
                                             const Fr& fold, Fr (&acc)[3]) {
  Fr x0, x1;
  round_pair<kFold>(tabs[0], j, q, fold, x0, x1);
  const Fr a0 = x0, a2 = fr_sub(fr_add(x0, x0), x1), da = fr_sub(x1, x0);
  round_pair<kFold>(tabs[1], j, q, fold, x0, x1);
  const Fr ab = fr_mul_call(a0, x0);
  const Fr ab2 = fr_mul_call(a2, fr_sub(fr_add(x0, x0), x1));
  const Fr dab = fr_mul_call(da, fr_sub(x1, x0));
  round_pair<kFold>(tabs[2], j, q, fold, x0, x1);
  const Fr t0 = fr_sub(ab, x0), t1 = fr_sub(ab2, fr_sub(fr_add(x0, x0), x1));
  round_pair<kFold>(tabs[3], j, q, fold, x0, x1);
  acc[0] = fr_add(acc[0], fr_mul_call(x0, t0));
  acc[1] = fr_add(acc[1], fr_mul_call(fr_sub(fr_add(x0, x0), x1), t1));
  acc[2] = fr_add(acc[2], fr_mul_call(fr_sub(x1, x0), dab));
}

}  // namespace pk
