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

// A synthetic R1CS with verifier challenges (pkg_synthetic_r1cs_dual): the
// single-commitment instance as w1, then a w2 of challenges and of products
// challenge x (w1 terms), the shape of a LogUp argument's challenge-dependent
// witnesses.  No reference counterpart (the reference compiles such circuits
// from Noir programs with lookups).
extern "C" int pkg_synthetic_r1cs_dual(uint64_t seed, size_t nc1, size_t ni, size_t nchal,
                                       size_t rows2, uint64_t* row_ptr[3], uint32_t* cols[3],
                                       uint64_t* vals[3], size_t nnz_out[3], uint64_t* witness,
                                       size_t* offsets) {
  PK_REQUIRE(nchal == 0 || offsets, "null offsets");
  const size_t w1 = 1 + ni + nc1, w2 = nchal + rows2;
  PK_REQUIRE(w1 + w2 < (size_t(1) << 32), "too many witnesses for u32 columns");
  int rc = pkg_synthetic_r1cs(seed, nc1, ni, row_ptr, cols, vals, nnz_out, witness);
  if (rc) return rc;
  memset(witness + 4 * w1, 0, 32 * w2);
  // challenge j at w2 offset j * floor(w2 / nchal), the products at the
  // other offsets in order
  const size_t stride = nchal ? w2 / nchal : 0;
  for (size_t j = 0; j < nchal; j++) offsets[j] = j * stride;
  SplitMix64 rng{seed ^ 0xd1b54a32d192ed03ULL};
  std::vector<uint64_t> coef(4 * 2 * (rows2 ? rows2 : 1));
  if ((rc = pkg_sample_fr(seed + 2, 2 * rows2, coef.data(), 1))) return rc;
  const HostFr one = HostFr::one();
  size_t ea = nnz_out[0], eb = nnz_out[1], used = 0, next = 0, j = 0;
  for (size_t i = 0; i < rows2; i++) {
    const size_t row = nc1 + i;
    // A: the challenge i mod nchal (the constant w[0] without challenges)
    cols[0][ea] = (uint32_t)(nchal ? w1 + offsets[i % nchal] : 0);
    memcpy(vals[0] + 4 * ea, one.l, 32);
    row_ptr[0][row + 1] = ++ea;
    // B: 1-2 uniform w1 columns
    const int kb = 1 + (int)rng.below(2);
    for (int q = 0; q < kb; q++) {
      cols[1][eb] = (uint32_t)rng.below(w1);
      memcpy(vals[1] + 4 * eb, coef.data() + 4 * used++, 32);
      eb++;
    }
    row_ptr[1][row + 1] = eb;
    // C: the next w2 offset that holds no challenge
    while (j < nchal && offsets[j] == next) {
      next++;
      j++;
    }
    cols[2][row] = (uint32_t)(w1 + next);
    memcpy(vals[2] + 4 * row, one.l, 32);
    row_ptr[2][row + 1] = row + 1;
    next++;
  }
  nnz_out[0] = ea;
  nnz_out[1] = eb;
  nnz_out[2] = nc1 + rows2;
  return PKG_OK;
}

// The caller-side solve of that instance's w2 (host): the challenges at
// their offsets, then for rows first_row.. in order w[C col] = (A w)(B w).
extern "C" int pkg_synthetic_dual_solve(size_t num_constraints, size_t first_row,
                                        const uint64_t* const row_ptr[3],
                                        const uint32_t* const cols[3],
                                        const uint64_t* const vals[3], size_t w1_size,
                                        const size_t* offsets, size_t nchal,
                                        const uint64_t* challenges, uint64_t* witness) {
  PK_REQUIRE(row_ptr && cols && vals && witness, "null pointer");
  PK_REQUIRE(nchal == 0 || (offsets && challenges), "null challenges");
  for (size_t j = 0; j < nchal; j++)
    memcpy(witness + 4 * (w1_size + offsets[j]), challenges + 4 * j, 32);
  for (size_t row = first_row; row < num_constraints; row++) {
    HostFr dot[2];
    for (int k = 0; k < 2; k++) {
      HostFr acc = HostFr::zero();
      for (uint64_t e = row_ptr[k][row]; e < row_ptr[k][row + 1]; e++)
        acc = HostFr::add(acc, HostFr::mul(HostFr::from_limbs(vals[k] + 4 * e),
                                           HostFr::from_limbs(witness + 4 * (size_t)cols[k][e])));
      dot[k] = acc;
    }
    const HostFr w = HostFr::mul(dot[0], dot[1]);
    memcpy(witness + 4 * (size_t)cols[2][row_ptr[2][row]], w.l, 32);
  }
  return PKG_OK;
}
