// synthetic.cu -- host-side generator of the synthetic satisfiable R1CS used
// by the prove benchmark and the parity tests (see pkg_synthetic_r1cs).
#include <cstring>
#include <vector>

#include "fr_host.hpp"
#include "pk_common.cuh"

namespace pk {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

}  // namespace pk

using namespace pk;

extern "C" int pkg_synthetic_r1cs(uint64_t seed, size_t nc, size_t ni, uint64_t* row_ptr[3],
                                  uint32_t* cols[3], uint64_t* vals[3], size_t nnz_out[3],
                                  uint64_t* witness) {
  PK_REQUIRE(row_ptr && cols && vals && nnz_out && witness, "null pointer");
  for (int k = 0; k < 3; k++) PK_REQUIRE(row_ptr[k] && cols[k] && vals[k], "null matrix array");
  PK_REQUIRE(ni + nc + 1 < (size_t(1) << 32), "too many witnesses for u32 columns");
  const size_t nw = 1 + ni + nc;
  SplitMix64 rng{seed};
  // structure first: counts and columns
  std::vector<uint8_t> ka(nc), kb(nc);
  size_t total = 0;
  for (size_t i = 0; i < nc; i++) {
    ka[i] = (uint8_t)(1 + rng.below(3));
    kb[i] = (uint8_t)(1 + rng.below(3));
    total += ka[i] + kb[i];
  }
  std::vector<uint64_t> coef(4 * (total ? total : 1));
  int rc = pkg_sample_fr(seed + 1, total, coef.data(), 1);
  if (rc) return rc;
  // inputs
  HostFr one = HostFr::one();
  memcpy(witness, one.l, 32);
  rc = pkg_sample_fr(seed, ni, witness + 4, 1);
  if (rc) return rc;
  size_t ea = 0, eb = 0, used = 0;
  row_ptr[0][0] = row_ptr[1][0] = row_ptr[2][0] = 0;
  for (size_t i = 0; i < nc; i++) {
    const uint64_t hi = ni + i + 1;  // columns in [0, ni + i]
    HostFr dot[2];
    for (int m = 0; m < 2; m++) {
      const int k = m == 0 ? ka[i] : kb[i];
      size_t& e = m == 0 ? ea : eb;
      HostFr acc = HostFr::zero();
      for (int j = 0; j < k; j++) {
        uint32_t col = (uint32_t)rng.below(hi);
        cols[m][e] = col;
        memcpy(vals[m] + 4 * e, coef.data() + 4 * used, 32);
        acc = HostFr::add(acc, HostFr::mul(HostFr::from_limbs(coef.data() + 4 * used),
                                           HostFr::from_limbs(witness + 4 * col)));
        used++;
        e++;
      }
      row_ptr[m][i + 1] = e;
      dot[m] = acc;
    }
    const size_t out_col = ni + 1 + i;
    cols[2][i] = (uint32_t)out_col;
    memcpy(vals[2] + 4 * i, one.l, 32);
    row_ptr[2][i + 1] = i + 1;
    HostFr w = HostFr::mul(dot[0], dot[1]);
    memcpy(witness + 4 * out_col, w.l, 32);
  }
  nnz_out[0] = ea;
  nnz_out[1] = eb;
  nnz_out[2] = nc;
  (void)nw;
  return PKG_OK;
}
