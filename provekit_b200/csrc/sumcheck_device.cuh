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

}  // namespace pk
