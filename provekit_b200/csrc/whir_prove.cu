// whir_prove.cu -- the WHIR prover's round loop, resident in HBM.
//
// The whir crate's prover (called from provekit/prover/src/whir_r1cs.rs:295-301,
// 378-414) is not vendored with the reference.  This loop produces the proof
// that the reference's Go verifier walks (runWhir,
// recursive-verifier/app/circuit/whir.go:587-724), for linear statements
// <a_k, c> = v_k about a committed coefficient vector c:
//
//   values v_k; combination randomness; k sumcheck rounds over
//   f^ = zeta(c) (subset sums: the hypercube evaluations of the multilinear
//   polynomial with coefficients c) and w = mobius^T(sum gamma^j a_j) plus
//   gamma^j eq(expand(z_j), .) for the commitment's OOD points;
//   per round: fold the coefficients, commit them (RS encode + Skyscraper
//   tree), OOD answers, PoW, STIR queries opened in the previous codeword,
//   their eq constraints added to w, k sumcheck rounds;
//   final: the remaining coefficients, PoW, STIR openings, sumcheck.
//
// Every table, codeword and tree stays on the device.  The host holds only the
// transcript: it reads back the three sums of each sumcheck round, the roots,
// the OOD answers, the PoW nonce and the opened rows and paths, which are the
// proof, and sends back the challenges as kernel parameters.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "fr_lazy.cuh"
#include "internal.cuh"
#include "pk_common.cuh"
#include "reduce.cuh"

namespace pk {

static_assert(sizeof(HostFr) == 32, "vectors of HostFr are arrays of 4 x u64 limbs");

// ---- subset transforms ----------------------------------------------------
// Zeta: v[b | 2^i] += v[b]; mobius^T: v[b] -= v[b | 2^i], over every index
// bit i.  A pass covers bits [lo, lo + nb): each CTA stages a tile of 2^nb
// rows (those bits) x 2^logw consecutive indices (the low bits, for
// coalesced 32-byte runs) in shared memory as two planes of 16-byte halves,
// runs its nb stages of additions there and writes the tile back.  The
// transform is memory-bound, so the pass count is what costs: a tile of
// kSubsetTile entries takes 10 bits in the first pass and 7 in each later
// one (21 bits: 3 passes).
constexpr int kSubsetLogTile = 10;
constexpr int kSubsetTile = 1 << kSubsetLogTile;  // Fr per CTA (32 KiB)
constexpr int kSubsetLogW = 3;                    // 8 consecutive indices after the first pass

__device__ __forceinline__ Fr tile_load(const uint4* t0, const uint4* t1, int e) {
  const uint4 a = t0[e], b = t1[e];
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}

__device__ __forceinline__ void tile_store(uint4* t0, uint4* t1, int e, const Fr& x) {
  t0[e] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  t1[e] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

template <bool kZeta>
__global__ void __launch_bounds__(256) subset_tile_kernel(uint64_t* __restrict__ v, int lo, int nb,
                                                          int logw) {
  __shared__ uint4 t0[kSubsetTile], t1[kSubsetTile];
  const int E = 1 << (nb + logw), W = 1 << logw;
  // this CTA: a block of W low indices (of 2^(lo - logw)) and a high part
  const size_t lblocks_log = (size_t)(lo - logw);
  const size_t lb = blockIdx.x & ((size_t(1) << lblocks_log) - 1);
  const size_t hi = (size_t)blockIdx.x >> lblocks_log;
  const size_t base = (hi << (lo + nb)) | (lb << logw);
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    const uint4* q = reinterpret_cast<const uint4*>(
        v + 4 * (base + ((size_t)(e >> logw) << lo) + (e & (W - 1))));
    t0[e] = q[0];
    t1[e] = q[1];
  }
  __syncthreads();
#pragma unroll 1
  for (int b = 0; b < nb; b++) {
    for (int p = threadIdx.x; p < E / 2; p += blockDim.x) {
      const int c = p & (W - 1), rp = p >> logw;
      const int r = ((rp >> b) << (b + 1)) | (rp & ((1 << b) - 1));  // row with bit b clear
      const int e0 = (r << logw) | c, e1 = ((r | (1 << b)) << logw) | c;
      const Fr x0 = tile_load(t0, t1, e0), x1 = tile_load(t0, t1, e1);
      if (kZeta)
        tile_store(t0, t1, e1, fr_add(x1, x0));
      else
        tile_store(t0, t1, e0, fr_sub(x0, x1));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    uint4* q = reinterpret_cast<uint4*>(v + 4 * (base + ((size_t)(e >> logw) << lo) + (e & (W - 1))));
    q[0] = t0[e];
    q[1] = t1[e];
  }
}

template <bool kZeta>
static int subset_transform_device(uint64_t* v, unsigned n, cudaStream_t s) {
  for (unsigned lo = 0; lo < n;) {
    const int logw = lo == 0 ? 0 : (int)std::min<unsigned>(lo, kSubsetLogW);
    const int nb = (int)std::min<unsigned>(kSubsetLogTile - logw, n - lo);
    const size_t ctas = size_t(1) << (n - nb - logw);
    subset_tile_kernel<kZeta><<<(unsigned)ctas, 256, 0, s>>>(v, (int)lo, nb, logw);
    PK_CHECK_LAUNCH("subset_tile_kernel");
    lo += nb;
  }
  return PKG_OK;
}

// ---- covector combination and table folds ----------------------------------
constexpr int kMaxCovectors = 16;
struct CovParams {
  const uint64_t* cov;
  size_t stride;  // Fr between covectors
  int ncov;
  uint32_t coef[kMaxCovectors][8];
};

// w[b] = sum_a coef_a cov[a][b]
__global__ void combine_covectors_kernel(uint64_t* __restrict__ w, size_t n,
                                         const __grid_constant__ CovParams P) {
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < n;
       b += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_zero();
    for (int a = 0; a < P.ncov; a++) {
      Fr c;
#pragma unroll
      for (int i = 0; i < 8; i++) c.v[i] = P.coef[a][i];
      acc = fr_add(acc, fr_mul_f64(c, fr_load_ro(P.cov, (size_t)a * P.stride + b)));
    }
    fr_store(w, b, acc);
  }
}

// The same sum with the products accumulated unreduced and reduced once per
// entry (fr_lazy.cuh); the coefficients carry a factor 2^8 (see
// combine_covectors).
__global__ void __launch_bounds__(128, 4) combine_covectors_lazy_kernel(
    uint64_t* __restrict__ w, size_t n, const __grid_constant__ CovParams P) {
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < n;
       b += (size_t)gridDim.x * blockDim.x) {
    lazy::Acc acc;
    acc.zero();
    for (int a = 0; a < P.ncov; a++) {
      Fr c;
#pragma unroll
      for (int i = 0; i < 8; i++) c.v[i] = P.coef[a][i];
      acc.mac(c, fr_load_ro(P.cov, (size_t)a * P.stride + b));
    }
    fr_store(w, b, acc.finish());  // kMaxCovectors < kCarryEvery: no carry needed
  }
}

static_assert(kMaxCovectors < lazy::kCarryEvery, "one carry-free lazy sum per entry");

// w = sum_a coefs[a] cov[a] over n entries (coefs host, Montgomery form):
// the lazy sum from four covectors on, where its one reduction per entry
// costs less than the products it saves.
static int combine_covectors(uint64_t* w, size_t n, const uint64_t* cov, size_t stride,
                             const HostFr* coefs, size_t ncov, cudaStream_t s) {
  CovParams P;
  memset(&P, 0, sizeof P);
  P.cov = cov;
  P.stride = stride;
  P.ncov = (int)ncov;
  const bool use_lazy = ncov >= 4;
  const HostFr m8 = HostFr::from_limbs(lazy::kMont2e8);
  for (size_t a = 0; a < ncov; a++) {
    const HostFr c = use_lazy ? HostFr::mul(coefs[a], m8) : coefs[a];
    memcpy(P.coef[a], c.l, 32);
  }
  if (use_lazy) {
    const int grid = (int)std::max<size_t>(
        1, std::min<size_t>((n + 127) / 128, (size_t)sm_count() * 4 * 8));
    combine_covectors_lazy_kernel<<<grid, 128, 0, s>>>(w, n, P);
    PK_CHECK_LAUNCH("combine_covectors_lazy_kernel");
  } else {
    combine_covectors_kernel<<<ew_grid(n), 256, 0, s>>>(w, n, P);
    PK_CHECK_LAUNCH("combine_covectors_kernel");
  }
  return PKG_OK;
}

// t[i] += r (t[i + h] - t[i]) for both tables: bind the top variable.
__global__ void fold_tables_kernel(uint64_t* __restrict__ f, uint64_t* __restrict__ w, size_t h,
                                   Fr r) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < h;
       i += (size_t)gridDim.x * blockDim.x) {
    const Fr f0 = fr_load(f, i), w0 = fr_load(w, i);
    fr_store(f, i, fr_add(f0, fr_mul_f64(r, fr_sub(fr_load(f, i + h), f0))));
    fr_store(w, i, fr_add(w0, fr_mul_f64(r, fr_sub(fr_load(w, i + h), w0))));
  }
}

// ---- parameters -------------------------------------------------------------
static unsigned rows_log(const pkg_whir_params* p, unsigned r) {
  return p->num_variables + p->log_inv_rate - p->folding_factor - r;
}

// Fr per opened row of codeword r: the first holds every batched polynomial.
static size_t row_fr(const pkg_whir_params* p, unsigned r) {
  return (size_t(1) << p->folding_factor) * (r == 0 ? p->batch_size : 1);
}

static bool params_ok(const pkg_whir_params* p) {
  if (!p) return false;
  const unsigned n = p->num_variables, k = p->folding_factor, R = p->num_rounds;
  if (k < 1 || k > 6 || n > 30 || R > PKG_WHIR_MAX_ROUNDS) return false;
  if (p->log_inv_rate < 1 || p->log_inv_rate > 8) return false;
  if ((R + 1) * k + p->final_vars != n) return false;
  if (p->ood_samples > 4 || p->pow_bits > 27 || p->final_pow_bits > 27) return false;
  if (p->batch_size != 1 && p->batch_size != 2 && p->batch_size != 4) return false;
  if (n + p->log_inv_rate < k + R + 1) return false;
  for (unsigned r = 0; r <= R; r++)
    if (p->queries[r] < 1 || p->queries[r] > 4096) return false;
  return true;
}

// ---- host-side protocol pieces -----------------------------------------------
static HostFr absorb_squeeze(pkg_transcript* t, const HostFr* msgs, size_t n) {
  for (size_t i = 0; i < n; i++) pkg_transcript_absorb(t, msgs[i].l);
  HostFr r;
  pkg_transcript_squeeze(t, r.l);
  return r;
}

static std::vector<HostFr> powers_of(const HostFr& g, size_t n) {
  std::vector<HostFr> out(n);
  if (n) out[0] = HostFr::one();
  for (size_t i = 1; i < n; i++) out[i] = HostFr::mul(out[i - 1], g);
  return out;
}


static void pow_threshold(unsigned bits, uint64_t thr[4]) {
  memcpy(thr, HostFr::P, 32);
  for (unsigned s = 0; s < bits; s++) {
    thr[0] = (thr[0] >> 1) | (thr[1] << 63);
    thr[1] = (thr[1] >> 1) | (thr[2] << 63);
    thr[2] = (thr[2] >> 1) | (thr[3] << 63);
    thr[3] >>= 1;
  }
}

// A stream-ordered allocation from the library pool that can be handed on.
struct PoolBuf {
  void* ptr = nullptr;
  cudaStream_t s = nullptr;
  PoolBuf() = default;
  PoolBuf(const PoolBuf&) = delete;
  PoolBuf& operator=(const PoolBuf&) = delete;
  int alloc(size_t bytes, cudaStream_t stream) {
    reset();
    s = stream;
    cudaMemPool_t pool = lib_pool();
    if (!pool) {
      set_last_error("could not create the library memory pool");
      return PKG_ERR_CUDA;
    }
    PK_CUDA(cudaMallocFromPoolAsync(&ptr, bytes, pool, s));
    return PKG_OK;
  }
  void reset() {
    if (ptr) cudaFreeAsync(ptr, s);
    ptr = nullptr;
  }
  void swap(PoolBuf& o) {
    std::swap(ptr, o.ptr);
    std::swap(s, o.s);
  }
  ~PoolBuf() { reset(); }
  template <class T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

// Host wall-clock of the calling thread's last WHIR prove, per phase
// (pkg_last_whir_stages).  Phases that end without a synchronisation leave
// their device time to the next one that synchronises.
thread_local double g_whir_ms[PKG_WHIR_STAGES];

struct PhaseTimer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  int k;
  explicit PhaseTimer(int stage) : k(stage) {}
  ~PhaseTimer() {
    g_whir_ms[k] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                        .count();
  }
};

#define PK_TRY(call)          \
  do {                        \
    const int _rc = (call);   \
    if (_rc) return _rc;      \
  } while (0)

// The proof's STIR openings feed no transcript value, so their copies run
// behind the proof's later steps into the thread's pinned stage
// (pinned_stage: one grow-only buffer per host thread and device, whose
// event marks the last copy into it, so a proof that ended early cannot leave
// copies landing in the next one's openings) and are moved into the proof
// after its last synchronisation.

class WhirProver {
 public:
  WhirProver(const pkg_whir_params* p, pkg_transcript* t, cudaStream_t s, uint64_t* proof)
      : p_(p), t_(t), s_(s), out_(proof) {}

  int run(const uint64_t* coeffs, const uint64_t* codeword, const uint8_t* layers,
          const uint64_t* ood_points, const uint64_t* covectors, size_t ncov,
          const uint64_t* values, uint64_t* hat);
  size_t words() const { return pos_; }

 private:
  void put(const HostFr& x) {
    memcpy(out_ + pos_, x.l, 32);
    pos_ += 4;
  }
  int sumcheck_phase(unsigned rounds, std::vector<HostFr>& rands, bool last = false);
  // Moves the staged openings into the proof.  Only call it when the stream
  // has passed a synchronisation since their copies were enqueued.
  void place_openings() {
    for (const Placement& pl : place_) memcpy(out_ + pl.word, stage_->buf + pl.src, pl.bytes);
    place_.clear();
  }
  int pow_step(unsigned bits);
  int stir_step(size_t q, size_t L, size_t row, const uint64_t* cw, const uint8_t* layers,
                std::vector<uint64_t>& idx);
  int add_constraints(const std::vector<HostFr>& points, unsigned nv,
                      const std::vector<HostFr>& coefs);

  const pkg_whir_params* p_;
  pkg_transcript* t_;
  cudaStream_t s_;
  uint64_t* out_;
  size_t pos_ = 0;
  // STIR openings: staged copies and where each lands in the proof
  struct Placement {
    size_t word, src, bytes;
  };
  PinnedStage* stage_ = nullptr;
  size_t stage_off_ = 0;
  std::vector<Placement> place_;
  uint64_t* E_ = nullptr;  // f^ table (live size size_)
  uint64_t* w_ = nullptr;  // weight table
  size_t size_ = 0;
};

// Tables of at most this many entries run the proof's last sumcheck on the
// host (a device round there is launch and round-trip latency).
constexpr size_t kHostTailEntries = 64;

// whir_round_kernel on host tables: fold the top variable by fold (if any,
// halving size), then h(0), h(1), h(2) of sum_b f(X, b) w(X, b).
static void host_whir_round(std::vector<HostFr>& f, std::vector<HostFr>& w, size_t& size,
                            const HostFr* fold, uint64_t out[12]) {
  if (fold) {
    const size_t h = size / 2;
    for (auto* t : {&f, &w})
      for (size_t j = 0; j < h; j++)
        (*t)[j] = HostFr::add((*t)[j], HostFr::mul(*fold, HostFr::sub((*t)[j + h], (*t)[j])));
    size = h;
  }
  const size_t q = size / 2;
  HostFr h0 = HostFr::zero(), h1 = HostFr::zero(), h2 = HostFr::zero();
  for (size_t j = 0; j < q; j++) {
    const HostFr f0 = f[j], f1 = f[j + q], w0 = w[j], w1 = w[j + q];
    h0 = HostFr::add(h0, HostFr::mul(f0, w0));
    h1 = HostFr::add(h1, HostFr::mul(f1, w1));
    h2 = HostFr::add(h2, HostFr::mul(HostFr::sub(HostFr::add(f1, f1), f0),
                                     HostFr::sub(HostFr::add(w1, w1), w0)));
  }
  memcpy(out, h0.l, 32);
  memcpy(out + 4, h1.l, 32);
  memcpy(out + 8, h2.l, 32);
}

// k rounds of the weighted sumcheck (runWhirSumcheckRounds,
// circuit/whir_utilities.go:103-126): send h(0), h(1), h(2), draw r.  The fold
// by r rides on the next round's kernel; the last one is done here.  The
// proof's last phase (last: nothing reads the tables afterwards) runs on
// the host when its tables are small.
int WhirProver::sumcheck_phase(unsigned rounds, std::vector<HostFr>& rands, bool last) {
  rands.clear();
  rands.reserve(rounds);
  if (last && rounds && size_ <= kHostTailEntries) {
    std::vector<HostFr> f(size_), w(size_);
    const HostRead reads[2] = {{f[0].l, E_, 32 * size_}, {w[0].l, w_, 32 * size_}};
    PK_TRY(read_small(reads, 2, s_));
    size_t size = size_;
    for (unsigned i = 0; i < rounds; i++) {
      uint64_t h[12];
      host_whir_round(f, w, size, i ? &rands.back() : nullptr, h);
      memcpy(out_ + pos_, h, 96);
      pos_ += 12;
      HostFr hs[3] = {HostFr::from_limbs(h), HostFr::from_limbs(h + 4), HostFr::from_limbs(h + 8)};
      rands.push_back(absorb_squeeze(t_, hs, 3));
    }
    return PKG_OK;
  }
  const uint64_t* pending = nullptr;
  HostFr r;
  for (unsigned i = 0; i < rounds; i++) {
    uint64_t h[12];
    PK_TRY(pkg_whir_sumcheck_round(E_, w_, size_, pending, h, reinterpret_cast<pkg_stream_t>(s_)));
    if (pending) size_ /= 2;
    memcpy(out_ + pos_, h, 96);
    pos_ += 12;
    HostFr hs[3] = {HostFr::from_limbs(h), HostFr::from_limbs(h + 4), HostFr::from_limbs(h + 8)};
    r = absorb_squeeze(t_, hs, 3);
    rands.push_back(r);
    pending = rands.back().l;
  }
  if (pending) {
    Fr rf;
    memcpy(rf.v, rands.back().l, 32);
    fold_tables_kernel<<<ew_grid(size_ / 2), 256, 0, s_>>>(E_, w_, size_ / 2, rf);
    PK_CHECK_LAUNCH("fold_tables_kernel");
    size_ /= 2;
  }
  return PKG_OK;
}

// RunPoW (circuit/whir.go:726-735): a challenge from the transcript, the
// smallest nonce below the threshold, the nonce back into the transcript.
int WhirProver::pow_step(unsigned bits) {
  HostFr cm;
  pkg_transcript_squeeze(t_, cm.l);
  const HostFr c = HostFr::from_mont(cm);
  uint64_t thr[4], nonce = 0;
  pow_threshold(bits, thr);
  PK_TRY(pow_solve_device(c.l, thr, s_, &nonce));
  out_[pos_++] = nonce;
  const HostFr nm = HostFr::from_u64(nonce);
  pkg_transcript_absorb(t_, nm.l);
  return PKG_OK;
}

// getStirChallenges (circuit/whir_utilities.go:49-78) on a codeword of L
// rows, then each queried row and its authentication path into the proof
// (copied into the staging buffer now, placed at the end of the proof).
int WhirProver::stir_step(size_t q, size_t L, size_t K, const uint64_t* cw, const uint8_t* layers,
                          std::vector<uint64_t>& idx) {
  // K: Fr per row (the batch's width for the first codeword)
  const int depth = log2_exact(L);
  const size_t nb = (size_t)(depth + 7) / 8;
  std::vector<uint8_t> bytes(q * nb + 1);
  PK_TRY(pkg_transcript_squeeze_bytes(t_, bytes.data(), q * nb));
  idx.assign(q, 0);
  PK_TRY(pkg_stir_indices(bytes.data(), L, q, idx.data()));
  const size_t row_bytes = 32 * K, path_bytes = 32 * (size_t)depth;
  PK_REQUIRE(stage_off_ + q * (row_bytes + path_bytes) <= stage_->cap,
             "opening staging too small");
  uint8_t* rows = stage_->buf + stage_off_;
  uint8_t* paths = rows + q * row_bytes;
  PK_TRY(open_rows_device(cw, K, L, layers, idx.data(), q, reinterpret_cast<uint64_t*>(rows),
                          paths, s_, false));
  PK_CUDA(cudaEventRecord(stage_->copied, s_));
  for (size_t i = 0; i < q; i++) {
    place_.push_back({pos_, stage_off_ + i * row_bytes, row_bytes});
    pos_ += 4 * K;
    place_.push_back({pos_, stage_off_ + q * row_bytes + i * path_bytes, path_bytes});
    pos_ += 4 * (size_t)depth;
  }
  stage_off_ += q * (row_bytes + path_bytes);
  return PKG_OK;
}

// w += sum_j coefs_j eq(expand(points_j), .) on the live nv-variable table.
int WhirProver::add_constraints(const std::vector<HostFr>& points, unsigned nv,
                                const std::vector<HostFr>& coefs) {
  // points and coefs are pageable: staged before the copies return, no
  // sync; the points are expanded on the device
  if (points.empty()) return PKG_OK;
  return eq_accumulate_device(w_, nv, points[0].l, coefs[0].l, points.size(), s_, false, false);
}

int WhirProver::run(const uint64_t* coeffs, const uint64_t* codeword, const uint8_t* layers,
                    const uint64_t* ood_points, const uint64_t* covectors, size_t ncov,
                    const uint64_t* values, uint64_t* hat) {
  memset(g_whir_ms, 0, sizeof g_whir_ms);
  const unsigned n = p_->num_variables, k = p_->folding_factor, R = p_->num_rounds;
  const unsigned o = p_->ood_samples;
  const size_t N = size_t(1) << n, K = size_t(1) << k;
  const pkg_stream_t ps = reinterpret_cast<pkg_stream_t>(s_);
  {
    // every round's openings: rows of row_fr Fr and paths of rows_log digests
    size_t stage_bytes = 32;
    for (unsigned r = 0; r <= R; r++)
      stage_bytes += (size_t)p_->queries[r] * 32 * (row_fr(p_, r) + rows_log(p_, r));
    PK_TRY(pinned_stage(stage_bytes, &stage_));
    stage_off_ = 0;
    place_.clear();
  }

  PoolBuf E, W, A, B, Cb, cw_own, lay_own, cw_next, lay_next;
  const unsigned nb = p_->batch_size;
  std::vector<HostFr> vals(ncov * nb);
  HostFr gamma;
  std::vector<HostFr> pw;
  // the batch's combination c = sum_i b^i f_i (b drawn at the commitment);
  // a single polynomial is c itself
  const uint64_t* poly = coeffs;
  {
  PhaseTimer pt(0);
  PK_TRY(W.alloc(32 * N, s_));
  PK_TRY(A.alloc(32 * (N >> k), s_));
  PK_TRY(B.alloc(32 * (N >> k), s_));
  w_ = W.as<uint64_t>();
  size_ = N;
  const std::vector<HostFr> bp =
      powers_of(nb > 1 ? HostFr::from_limbs(ood_points + 4 * o) : HostFr::one(), nb);
  if (nb > 1) {
    PK_TRY(Cb.alloc(32 * N, s_));
    PK_TRY(combine_covectors(Cb.as<uint64_t>(), N, coeffs, N, bp.data(), nb, s_));
    poly = Cb.as<uint64_t>();
  }
  if (hat && nb == 1) {
    E_ = hat;  // the caller's zeta(coeffs), folded in place from here on
  } else {
    PK_TRY(E.alloc(32 * N, s_));
    E_ = E.as<uint64_t>();
    PK_CUDA(cudaMemcpyAsync(E_, poly, 32 * N, cudaMemcpyDeviceToDevice, s_));
    PK_TRY(subset_transform_device<true>(E_, n, s_));
  }

  // the statement values, polynomial by polynomial, then the combination
  // randomness over (commitment OOD answers, values)
  for (unsigned i = 0; i < nb; i++)
    for (size_t a = 0; a < ncov; a++) {
      HostFr& v = vals[i * ncov + a];
      if (values)
        memcpy(v.l, values + 4 * (i * ncov + a), 32);
      else
        PK_TRY(pkg_dot(covectors + 4 * N * a, coeffs + 4 * N * i, N, v.l, ps));
      put(v);
    }
  gamma = absorb_squeeze(t_, vals.data(), ncov * nb);
  pw = powers_of(gamma, o + ncov);
  if (ncov) {
    PK_TRY(combine_covectors(w_, N, covectors, N, pw.data() + o, ncov, s_));
    PK_TRY(subset_transform_device<false>(w_, n, s_));
  } else {
    PK_CUDA(cudaMemsetAsync(w_, 0, 32 * N, s_));
  }
  if (o) {
    std::vector<HostFr> z(o), c(pw.begin(), pw.begin() + o);
    for (unsigned j = 0; j < o; j++) z[j] = HostFr::from_limbs(ood_points + 4 * j);
    PK_TRY(add_constraints(z, n, c));
  }
  }

  std::vector<HostFr> alpha;
  {
    PhaseTimer pt(1);
    PK_TRY(sumcheck_phase(k, alpha));
  }

  const uint64_t* f = poly;  // current polynomial's coefficients
  unsigned nv = n;
  const uint64_t* cw_r = codeword;
  const uint8_t* lay_r = layers;
  std::vector<uint64_t> idx;
  auto fold_into = [&](uint64_t* g) -> int {
    std::vector<HostFr> ra(alpha.rbegin(), alpha.rend());
    PK_TRY(pkg_whir_fold_coeffs(f, size_t(1) << nv, k, ra[0].l, g, ps));
    nv -= k;
    return PKG_OK;
  };
  for (unsigned r = 0; r < R; r++) {
    uint64_t* g = (r & 1) ? B.as<uint64_t>() : A.as<uint64_t>();
    const size_t Ln = size_t(1) << rows_log(p_, r + 1);
    {
      PhaseTimer pt(2);
      PK_TRY(fold_into(g));
      // commit the folded polynomial at the next rate
      PK_TRY(cw_next.alloc(32 * K * Ln, s_));
      PK_TRY(lay_next.alloc(32 * (2 * Ln - 1), s_));
      PK_TRY(pkg_whir_commit(g, size_t(1) << nv, k, p_->log_inv_rate + (r + 1) * (k - 1), nullptr,
                             0, PKG_LEAF_CANONICAL, cw_next.as<uint64_t>(), lay_next.as<uint8_t>(),
                             ps));
      // the previous round's openings (copied before that round's sumcheck
      // synchronised) go into the proof while the device encodes and hashes
      place_openings();
      HostFr root;
      PK_TRY(read_small(root.l, lay_next.as<uint8_t>() + 32 * (2 * Ln - 2), 32, s_));
      put(root);
      const HostFr root_m = HostFr::to_mont(root);
      pkg_transcript_absorb(t_, root_m.l);
    }
    // OOD samples of the folded polynomial
    std::vector<HostFr> points(o);
    {
      PhaseTimer pt(3);
      for (unsigned j = 0; j < o; j++) pkg_transcript_squeeze(t_, points[j].l);
      if (o) {
        std::vector<HostFr> ans(o);
        PK_TRY(pkg_poly_eval_many(g, size_t(1) << nv, points[0].l, o, ans[0].l, ps));
        for (unsigned j = 0; j < o; j++) {
          put(ans[j]);
          pkg_transcript_absorb(t_, ans[j].l);
        }
      }
    }
    if (p_->pow_bits) {
      PhaseTimer pt(4);
      PK_TRY(pow_step(p_->pow_bits));
    }
    // STIR queries on the previous codeword
    const size_t Lr = size_t(1) << rows_log(p_, r), q = p_->queries[r];
    {
      PhaseTimer pt(5);
      PK_TRY(stir_step(q, Lr, row_fr(p_, r), cw_r, lay_r, idx));
      std::vector<size_t> sidx(idx.begin(), idx.end());
      points.resize(o + q);
      PK_TRY(pkg_rs_evaluation_points(Lr, sidx.data(), q, points[o].l));
    }
    {
      PhaseTimer pt(6);
      HostFr gr;
      pkg_transcript_squeeze(t_, gr.l);
      PK_TRY(add_constraints(points, nv, powers_of(gr, o + q)));
    }
    {
      PhaseTimer pt(1);
      PK_TRY(sumcheck_phase(k, alpha));
    }
    // the new codeword becomes the one the next queries open
    f = g;
    cw_own.swap(cw_next);
    lay_own.swap(lay_next);
    cw_next.reset();
    lay_next.reset();
    cw_r = cw_own.as<uint64_t>();
    lay_r = lay_own.as<uint8_t>();
  }
  // the final polynomial in the clear
  {
    PhaseTimer pt(7);
    uint64_t* g = (R & 1) ? B.as<uint64_t>() : A.as<uint64_t>();
    PK_TRY(fold_into(g));
    const size_t nfin = size_t(1) << nv;
    std::vector<HostFr> fin(nfin);
    PK_TRY(read_small(fin[0].l, g, 32 * nfin, s_));
    for (size_t i = 0; i < nfin; i++) {
      put(fin[i]);
      pkg_transcript_absorb(t_, fin[i].l);
    }
  }
  if (p_->final_pow_bits) {
    PhaseTimer pt(4);
    PK_TRY(pow_step(p_->final_pow_bits));
  }
  {
    PhaseTimer pt(5);
    PK_TRY(stir_step(p_->queries[R], size_t(1) << rows_log(p_, R), row_fr(p_, R), cw_r, lay_r,
                     idx));
  }
  {
    PhaseTimer pt(1);
    std::vector<HostFr> rfin;
    PK_TRY(sumcheck_phase(nv, rfin, true));
    PK_CUDA(cudaStreamSynchronize(s_));
  }
  // the staged openings into their places
  place_openings();
  return PKG_OK;
}

int whir_prove_device(const pkg_whir_params* p, pkg_transcript* t, const uint64_t* coeffs,
                      const uint64_t* codeword, const uint8_t* layers, const uint64_t* ood_points,
                      const uint64_t* covectors, size_t ncov, const uint64_t* values,
                      uint64_t* hat, uint64_t* proof, cudaStream_t s) {
  WhirProver prover(p, t, s, proof);
  int rc = prover.run(coeffs, codeword, layers, ood_points, covectors, ncov, values, hat);
  if (rc) return rc;
  if (prover.words() != pkg_whir_proof_words(p, ncov)) {
    set_last_error("WHIR proof wrote %zu words, the layout has %zu", prover.words(),
                   pkg_whir_proof_words(p, ncov));
    return PKG_ERR_UNSUPPORTED;
  }
  return PKG_OK;
}

int subset_zeta_device(uint64_t* v, unsigned n, cudaStream_t s) {
  return subset_transform_device<true>(v, n, s);
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_whir_params_init(pkg_whir_params* p, unsigned n, unsigned k,
                                    unsigned log_inv_rate, unsigned security_bits,
                                    unsigned pow_bits) {
  PK_REQUIRE(p, "null params");
  PK_REQUIRE(k >= 1 && k <= 6 && n >= k && n <= 30, "unsupported n = %u, k = %u", n, k);
  PK_REQUIRE(log_inv_rate >= 1 && log_inv_rate <= 8, "log_inv_rate %u outside 1..8", log_inv_rate);
  PK_REQUIRE(pow_bits <= 27 && security_bits > pow_bits && security_bits <= 512,
             "unsupported security %u / pow %u", security_bits, pow_bits);
  memset(p, 0, sizeof *p);
  unsigned folds = n > 6 ? (n - 6 + k - 1) / k : 1;
  if (folds * k > n) folds = n / k;
  PK_REQUIRE(folds >= 1 && folds - 1 <= PKG_WHIR_MAX_ROUNDS, "too many rounds");
  p->num_variables = n;
  p->folding_factor = k;
  p->log_inv_rate = log_inv_rate;
  p->num_rounds = folds - 1;
  p->final_vars = n - folds * k;
  p->ood_samples = 1;
  p->pow_bits = pow_bits;
  p->final_pow_bits = pow_bits;
  p->batch_size = 1;
  for (unsigned r = 0; r <= p->num_rounds; r++) {
    const unsigned rate = log_inv_rate + r * (k - 1);
    const unsigned q = (2 * (security_bits - pow_bits) + rate - 1) / rate;
    p->queries[r] = std::min(q, 4096u);
  }
  PK_REQUIRE(params_ok(p), "parameters give a codeword of one row");
  return PKG_OK;
}

extern "C" size_t pkg_whir_commit_words(const pkg_whir_params* p) {
  return p ? 4 + 4 * (size_t)p->ood_samples * p->batch_size : 0;
}

extern "C" size_t pkg_whir_proof_words(const pkg_whir_params* p, size_t ncov) {
  if (!params_ok(p)) return 0;
  const size_t k = p->folding_factor;
  size_t w = 4 * ncov * p->batch_size + 12 * k;
  for (unsigned r = 0; r < p->num_rounds; r++)
    w += 4 + 4 * (size_t)p->ood_samples + (p->pow_bits ? 1 : 0) +
         (size_t)p->queries[r] * (4 * row_fr(p, r) + 4 * rows_log(p, r)) + 12 * k;
  const unsigned R = p->num_rounds;
  w += 4 * (size_t(1) << p->final_vars) + (p->final_pow_bits ? 1 : 0) +
       (size_t)p->queries[R] * (4 * row_fr(p, R) + 4 * rows_log(p, R)) +
       12 * (size_t)p->final_vars;
  return w;
}

extern "C" int pkg_subset_transform(uint64_t* v, unsigned n, int mode, pkg_stream_t stream) {
  PK_REQUIRE(n <= 34, "too many variables (%u)", n);
  PK_REQUIRE(mode == PKG_SUBSET_ZETA || mode == PKG_SUBSET_MOBIUS_T, "unknown mode %d", mode);
  PK_REQUIRE(v && aligned16(v), "null or unaligned table");
  return mode == PKG_SUBSET_ZETA ? subset_transform_device<true>(v, n, as_stream(stream))
                                 : subset_transform_device<false>(v, n, as_stream(stream));
}

extern "C" int pkg_whir_commit_ood(const pkg_whir_params* p, pkg_transcript* t,
                                   const uint64_t* coeffs, const uint8_t* layers,
                                   uint64_t* commit_words, uint64_t* ood_points,
                                   pkg_stream_t stream) {
  PK_REQUIRE(params_ok(p), "invalid WHIR parameters");
  PK_REQUIRE(t && coeffs && layers && commit_words && (ood_points || !p->ood_samples),
             "null pointer");
  PK_REQUIRE(aligned16(coeffs) && aligned16(layers), "device buffers must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  const size_t L = size_t(1) << rows_log(p, 0);
  HostFr root;
  {
    int rc = read_small(root.l, layers + 32 * (2 * L - 2), 32, s);
    if (rc) return rc;
  }
  PK_REQUIRE(root.is_canonical(), "root digest is not a canonical field element");
  const HostFr rm = HostFr::to_mont(root);
  pkg_transcript_absorb(t, rm.l);
  memcpy(commit_words, root.l, 32);
  const unsigned o = p->ood_samples;
  const size_t N = size_t(1) << p->num_variables;
  for (unsigned j = 0; j < o; j++) pkg_transcript_squeeze(t, ood_points + 4 * j);
  // f_i(z_j), polynomial by polynomial (parseBatchedCommitment,
  // recursive-verifier/app/circuit/mtUtilities.go:51-76)
  for (unsigned i = 0; o && i < p->batch_size; i++) {
    int rc = pkg_poly_eval_many(coeffs + 4 * N * i, N, ood_points, o, commit_words + 4 + 4 * o * i,
                                stream);
    if (rc) return rc;
  }
  for (unsigned j = 0; j < o * p->batch_size; j++)
    pkg_transcript_absorb(t, commit_words + 4 + 4 * j);
  if (p->batch_size > 1) pkg_transcript_squeeze(t, ood_points + 4 * o);  // batching challenge
  return PKG_OK;
}

extern "C" int pkg_whir_prove(const pkg_whir_params* p, pkg_transcript* t, const uint64_t* coeffs,
                              const uint64_t* codeword, const uint8_t* layers,
                              const uint64_t* ood_points, const uint64_t* covectors, size_t ncov,
                              uint64_t* proof, pkg_stream_t stream) {
  PK_REQUIRE(params_ok(p), "invalid WHIR parameters");
  PK_REQUIRE(ncov <= (size_t)kMaxCovectors, "at most %d covectors", kMaxCovectors);
  PK_REQUIRE(t && coeffs && codeword && layers && proof && (covectors || !ncov) &&
                 (ood_points || !p->ood_samples),
             "null pointer");
  PK_REQUIRE(aligned16(coeffs) && aligned16(codeword) && aligned16(layers) &&
                 (!ncov || aligned16(covectors)),
             "device buffers must be 16-byte aligned");
  return whir_prove_device(p, t, coeffs, codeword, layers, ood_points, covectors, ncov, nullptr,
                           nullptr, proof, as_stream(stream));
}

extern "C" int pkg_last_whir_stages(double ms[PKG_WHIR_STAGES]) {
  PK_REQUIRE(ms, "null output");
  memcpy(ms, g_whir_ms, sizeof g_whir_ms);
  return PKG_OK;
}
