// ntt.cu -- BN254 Fr NTT for sm_100a: the ntt crate's ntt_nr / intt_rn
// (ntt/src/ntt.rs:105-348) behind pkg_ntt_nr / pkg_intt_rn.
//
// Algorithm: the same radix-2 DIT, normal-in / bit-reversed-out transform as
// interleaved_ntt_nr (ntt/src/ntt.rs:150-248).  At global stage t there are
// 2^t groups; group k pairs element i with i + half and multiplies the odd
// element by roots[k] from the bit-reversed twiddle table
// (init_roots_reverse_ordered, ntt/src/ntt.rs:275-306).  Stages are fused into
// passes of K <= 10 stages: a pass owns independent 2^K-point sub-transforms
// ("lines": fixed top t row bits and fixed low row bits), stages each line in
// shared memory, and runs its K stages there, so global memory is read and
// written once per pass instead of once per stage.  Exact modular arithmetic
// makes the output bit-identical to the stage-by-stage CPU order.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "ntt_internal.cuh"
#include "host_stage.cuh"
#include "pk_common.cuh"

// Most stages per pass (a pass kernel exists for 1..9).  Eight: a 9-stage
// pass stages 2 x 2^8 x 11 doubles of twiddle digits (45 KiB) besides its
// 16 KiB tile, which holds it to 3 CTAs per SM; the whole proof's 18-stage
// witness encode ran 0.39 ms faster per proof as three 6-stage passes than as
// two 9-stage ones (18.65 vs 19.04 ms), and two 9-stage lines per CTA (512
// threads, 2 CTAs per SM) gained nothing.
#ifndef PK_NTT_KMAX
#define PK_NTT_KMAX 8
#endif
// Butterflies per thread per stage, log2 (the CTA has E / 2^(1 + this)
// threads, at least 32).  Two: 2^24 points in 5.01 ms against 5.14 ms with
// one (a CTA of 256 elements' worth of 128 threads, each with two
// independent products in flight per stage); four were slower (5.31 ms).
#ifndef PK_NTT_LOG_BPT
#define PK_NTT_LOG_BPT 1
#endif
// Elements per CTA, log2 (lines of 2^K elements: 2^(this - K) of them).
#ifndef PK_NTT_LOG_ELEMS
#define PK_NTT_LOG_ELEMS 9
#endif

namespace pk {

// ---------------------------------------------------------------------------
// Device-resident twiddle table (the NTTEngine, ntt/src/ntt.rs:24-95): one
// grow-only table per device, roots[bitrev(i)] = w_order^i for i < order/2.
// By the prefix property (ntt/src/ntt.rs:515-522) the first m/2 entries of
// the table for any order >= m are the order-m table.
// ---------------------------------------------------------------------------
struct RootsTable {
  uint64_t* d = nullptr;
  size_t order = 0;
  std::vector<uint64_t*> retired;
};
static std::mutex g_roots_mu;
static std::vector<RootsTable> g_roots;

__global__ void roots_kernel(uint64_t* __restrict__ roots, const uint64_t* __restrict__ w_lo,
                             const uint64_t* __restrict__ w_hi, int log_half, int s) {
  size_t n = size_t(1) << log_half;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr lo = fr_load_ro(w_lo, i & ((size_t(1) << s) - 1));
    Fr hi = fr_load_ro(w_hi, i >> s);
    Fr w = fr_mul(lo, hi);
    size_t r = __brevll((unsigned long long)i) >> (64 - log_half);
    fr_store(roots, r, w);
  }
}

int roots_reserve(size_t order, const uint64_t** out) {
  if (order < 1024) order = 1024;  // NTTEngine::new() size (ntt/src/ntt.rs:30-33)
  if (!is_pow2(order) || order > (size_t(1) << 28)) {
    set_last_error("twiddle order %zu is not a power of two <= 2^28", order);
    return PKG_ERR_INVALID_ARGUMENT;
  }
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_roots_mu);
  if ((int)g_roots.size() <= dev) g_roots.resize(dev + 1);
  RootsTable& tab = g_roots[dev];
  if (tab.order >= order) {
    *out = tab.d;
    return PKG_OK;
  }
  // Grow: build the order-`order` table.  Superseded tables stay allocated
  // (kept in `retired`) so that kernels already enqueued on any stream, or
  // pointers already handed to another thread, stay valid; by the prefix
  // property their total size is below the new table's.
  int log_half = log2_exact(order / 2);
  int s = (log_half + 1) / 2;
  size_t nlo = size_t(1) << s, nhi = size_t(1) << (log_half - s);
  HostFr w = HostFr::root_of_unity(order);
  std::vector<uint64_t> h_lo(4 * nlo), h_hi(4 * nhi);
  HostFr acc = HostFr::one();
  for (size_t i = 0; i < nlo; i++) {
    memcpy(&h_lo[4 * i], acc.l, 32);
    acc = HostFr::mul(acc, w);
  }
  HostFr step = acc;  // w^(2^s)
  acc = HostFr::one();
  for (size_t i = 0; i < nhi; i++) {
    memcpy(&h_hi[4 * i], acc.l, 32);
    acc = HostFr::mul(acc, step);
  }
  uint64_t *d_new = nullptr, *d_lo = nullptr, *d_hi = nullptr;
  PK_CUDA(cudaMalloc(&d_new, 32 * (order / 2)));
  cudaError_t e = cudaMalloc(&d_lo, 32 * nlo);
  if (e == cudaSuccess) e = cudaMalloc(&d_hi, 32 * nhi);
  if (e == cudaSuccess) e = cudaMemcpy(d_lo, h_lo.data(), 32 * nlo, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_hi, h_hi.data(), 32 * nhi, cudaMemcpyHostToDevice);
  // Built on a private stream and waited for, so the table is complete before
  // any caller (on any stream) can see the new pointer.
  cudaStream_t bs = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    int blocks = (int)std::min<size_t>((order / 2 + 255) / 256, (size_t)sm_count() * 16);
    roots_kernel<<<blocks, 256, 0, bs>>>(d_new, d_lo, d_hi, log_half, s);
    e = cudaGetLastError();
    count_launch();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(bs);
  if (bs) cudaStreamDestroy(bs);
  cudaFree(d_lo);
  cudaFree(d_hi);
  if (e != cudaSuccess) {
    cudaFree(d_new);
    return cuda_status(e, "twiddle table");
  }
  if (tab.d) tab.retired.push_back(tab.d);
  tab.d = d_new;
  tab.order = order;
  *out = tab.d;
  return PKG_OK;
}

// ---------------------------------------------------------------------------
// Pass kernel.
//
// Shared memory holds the CTA's E elements as two planes of 16-byte halves
// (plane 0: bytes 0-15 of every element, plane 1: bytes 16-31), so a warp
// touching consecutive elements reads consecutive 16-byte words.
//
// Row r of the transform (codeword position) has log2(N) bits.  A pass over
// global stages [t, t+K) splits r = (high : j : low) with high = top t bits,
// j = next K bits, low = remaining B bits.  With M interleaved columns, the
// element (r, c) sits at r*M + c; "line" = (high, u) with u = low*M + c in
// [0, U), U = 2^B * M, and line element j is at (high*2^K + j)*U + u.
// A CTA owns T consecutive lines.  Mode A (T divides U): the lines share
// `high` and are contiguous per j.  Mode B (U divides T, U a power of two):
// the CTA's lines cover a contiguous memory range.
// Stage s of the pass (global stage t+s) pairs j0 = grp*2h + pos with
// j0 + h (h = 2^(K-1-s)) and uses twiddle roots[(high << s) | grp].
// ---------------------------------------------------------------------------
// Element g of the RS-encode layout (see NttSource).
__device__ __forceinline__ Fr source_load(const NttSource& s, uint64_t g) {
  const uint64_t x = g % s.chunk;
  if (x < s.L * s.M) {
    const uint64_t row = x / s.M, col = x - row * s.M;
    return fr_load_ro(s.messages, col * s.L + row);
  }
  if (x - s.L * s.M < s.mask_len) return fr_load_ro(s.masks, x - s.L * s.M);
  return fr_zero();
}

// kModeB selects mode B at compile time.  In mode A every line of the CTA
// shares `high`, so stage s needs only the 2^s twiddles roots[(high << s) |
// grp]; they are converted to FP64 digits once per CTA into shared memory
// after the data tile (double-buffered across stages, 2 x 2^(K-1) x 11
// doubles) instead of once per butterfly.
template <int K, bool kSrc, bool kModeB>
__global__ void __launch_bounds__(512) ntt_pass_kernel(uint64_t* __restrict__ data,
                                                      const uint64_t* __restrict__ roots,
                                                      uint64_t U, int log_u, int T, int log_t,
                                                      int mode_b_unused, const NttSource src) {
  extern __shared__ uint4 sm[];
  constexpr int R = 1 << K;
  constexpr bool mode_b = kModeB;
  const int E = R * T;
  double* tw = reinterpret_cast<double*>(sm + 2 * E);
  constexpr int kTw = (R / 2) * 11;
  const uint64_t l0 = (uint64_t)blockIdx.x * T;
  uint64_t high_a = 0, u0 = 0;
  if (!mode_b) {
    high_a = l0 / U;
    u0 = l0 - high_a * U;
  }
  // ---- load ----
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    uint64_t g;
    int sidx;
    if (!mode_b) {
      int j = e >> log_t, ll = e & (T - 1);
      g = (high_a * R + j) * U + u0 + ll;
      sidx = j * T + ll;
    } else {
      int j = (e >> log_u) & (R - 1);
      int hl = e >> (log_u + K);
      int u = e & ((1 << log_u) - 1);
      g = (l0 >> log_u) * R * U + e;
      sidx = j * T + (hl << log_u) + u;
    }
    if (kSrc) {
      const Fr v = source_load(src, g);
      sm[sidx] = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
      sm[E + sidx] = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
    } else {
      const uint4* in = reinterpret_cast<const uint4*>(data + 4 * g);
      sm[sidx] = in[0];      // low 16 bytes: plane 0
      sm[E + sidx] = in[1];  // high 16 bytes: plane 1
    }
  }
  if (!kModeB && threadIdx.x == 0) f64::digits(fr_load_ro(roots, high_a), tw);  // stage 0
  __syncthreads();
  // ---- K radix-2 stages in shared memory ----
#pragma unroll 1
  for (int s = 0; s < K; s++) {
    const int log_h = K - 1 - s;
    for (int b = threadIdx.x; b < (E >> 1); b += blockDim.x) {
      int ll = b & (T - 1);
      int p = b >> log_t;
      int grp = p >> log_h;
      int pos = p & ((1 << log_h) - 1);
      int j0 = (grp << (log_h + 1)) + pos;
      int j1 = j0 + (1 << log_h);
      int i0 = j0 * T + ll, i1 = j1 * T + ll;
      Fr x0, x1;
      uint4 a = sm[i0], bb = sm[E + i0];
      x0.v[0] = a.x; x0.v[1] = a.y; x0.v[2] = a.z; x0.v[3] = a.w;
      x0.v[4] = bb.x; x0.v[5] = bb.y; x0.v[6] = bb.z; x0.v[7] = bb.w;
      a = sm[i1];
      bb = sm[E + i1];
      x1.v[0] = a.x; x1.v[1] = a.y; x1.v[2] = a.z; x1.v[3] = a.w;
      x1.v[4] = bb.x; x1.v[5] = bb.y; x1.v[6] = bb.z; x1.v[7] = bb.w;
      Fr m;
      if (kModeB) {
        const uint64_t high = (l0 + ll) >> log_u;
        m = fr_mul_f64(fr_load_ro(roots, (high << s) | (uint64_t)grp), x1);
      } else {
        m = fr_mul_f64_digits(tw + (s & 1) * kTw + 11 * grp, x1);
      }
      Fr y0 = fr_add(x0, m);
      Fr y1 = fr_sub(x0, m);
      sm[i0] = make_uint4(y0.v[0], y0.v[1], y0.v[2], y0.v[3]);
      sm[E + i0] = make_uint4(y0.v[4], y0.v[5], y0.v[6], y0.v[7]);
      sm[i1] = make_uint4(y1.v[0], y1.v[1], y1.v[2], y1.v[3]);
      sm[E + i1] = make_uint4(y1.v[4], y1.v[5], y1.v[6], y1.v[7]);
    }
    // next stage's twiddles into the other buffer: no thread reads it before
    // the barrier below, and its previous readers finished before the last one
    if (!kModeB && s + 1 < K) {
#pragma unroll 1
      for (int g = threadIdx.x; g < (2 << s); g += blockDim.x)
        f64::digits(fr_load_ro(roots, (high_a << (s + 1)) | (uint64_t)g),
                    tw + ((s + 1) & 1) * kTw + 11 * g);
    }
    __syncthreads();
  }
  // ---- store ----
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    uint64_t g;
    int sidx;
    if (!mode_b) {
      int j = e >> log_t, ll = e & (T - 1);
      g = (high_a * R + j) * U + u0 + ll;
      sidx = j * T + ll;
    } else {
      int j = (e >> log_u) & (R - 1);
      int hl = e >> (log_u + K);
      int u = e & ((1 << log_u) - 1);
      g = (l0 >> log_u) * R * U + e;
      sidx = j * T + (hl << log_u) + u;
    }
    uint4* dst = reinterpret_cast<uint4*>(data + 4 * g);
    dst[0] = sm[sidx];
    dst[1] = sm[E + sidx];
  }
}

typedef void (*PassFn)(uint64_t*, const uint64_t*, uint64_t, int, int, int, int, const NttSource);
template <bool kSrc, bool kModeB>
static PassFn pass_fn_t(int k) {
  switch (k) {
    case 1: return ntt_pass_kernel<1, kSrc, kModeB>;
    case 2: return ntt_pass_kernel<2, kSrc, kModeB>;
    case 3: return ntt_pass_kernel<3, kSrc, kModeB>;
    case 4: return ntt_pass_kernel<4, kSrc, kModeB>;
    case 5: return ntt_pass_kernel<5, kSrc, kModeB>;
    case 6: return ntt_pass_kernel<6, kSrc, kModeB>;
    case 7: return ntt_pass_kernel<7, kSrc, kModeB>;
    case 8: return ntt_pass_kernel<8, kSrc, kModeB>;
    default: return ntt_pass_kernel<9, kSrc, kModeB>;
  }
}
static PassFn pass_fn(int k, bool src, bool mode_b) {
  if (src) return mode_b ? pass_fn_t<true, true>(k) : pass_fn_t<true, false>(k);
  return mode_b ? pass_fn_t<false, true>(k) : pass_fn_t<false, false>(k);
}

static inline uint64_t pow2_part(uint64_t x) { return x & (~x + 1); }

// Run global stages [t_begin, t_end) of an N-point transform over M columns.
int ntt_stages(uint64_t* data, size_t N, size_t M, int t_begin, int t_end, const uint64_t* roots,
               cudaStream_t stream, const NttSource* src) {
  const int S = log2_exact(N);
  (void)S;
  const int kmax = PK_NTT_KMAX;
  int total = t_end - t_begin;
  if (total <= 0) return PKG_OK;
  int npasses = (total + kmax - 1) / kmax;
  int t = t_begin;
  for (int pi = 0; pi < npasses; pi++) {
    int K = (total - (t - t_begin) + (npasses - pi) - 1) / (npasses - pi);
    int B = log2_exact(N) - t - K;
    uint64_t U = (uint64_t(1) << B) * M;
    uint64_t num_lines = (uint64_t(1) << t) * U;
    // aim for 2^PK_NTT_LOG_ELEMS elements per CTA
    int log_tgt = K >= PK_NTT_LOG_ELEMS ? 0 : PK_NTT_LOG_ELEMS - K;
    uint64_t T = uint64_t(1) << log_tgt;
    if (T > num_lines) T = pow2_part(num_lines);
    int mode_b = 0;
    int log_u = 0;
    if (is_pow2(U) && U < T) {
      mode_b = 1;
      log_u = log2_exact(U);
    } else {
      uint64_t pu = pow2_part(U);
      if (T > pu) T = pu;
    }
    int log_t = log2_exact(T);
    uint64_t E = (uint64_t(1) << K) * T;
    int threads = (int)std::min<uint64_t>((E / 2) >> PK_NTT_LOG_BPT, 512);
    if (threads < 32) threads = 32;
    size_t smem = 32 * E + (mode_b ? 0 : sizeof(double) * 2 * 11 * (size_t(1) << (K - 1)));
    uint64_t grid = num_lines / T;
    const bool from_src = src != nullptr && pi == 0;
    PassFn fn = pass_fn(K, from_src, mode_b != 0);
    if (smem > 48 * 1024) {
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    NttSource s;
    memset(&s, 0, sizeof s);
    if (from_src) s = *src;
    fn<<<(unsigned)grid, threads, smem, stream>>>(data, roots, U, log_u, (int)T, log_t, mode_b, s);
    PK_CHECK_LAUNCH("ntt_pass_kernel");
    t += K;
  }
  return PKG_OK;
}

// Validation shared by the device and host forms (reference panics ->
// PKG_ERR_INVALID_ARGUMENT).  Returns 1 if there is nothing to do.
int ntt_validate(size_t len, size_t codeword_size, size_t num_groups, int* noop) {
  *noop = 0;
  if (codeword_size <= 1) {  // ntt/src/ntt.rs:161-163
    *noop = 1;
    return PKG_OK;
  }
  PK_REQUIRE(num_groups != 0 && len % num_groups == 0,
             "values.len() must be divisible by num_groups (len=%zu, num_groups=%zu)", len,
             num_groups);
  PK_REQUIRE(is_pow2(codeword_size), "codeword_size %zu is not a power of two", codeword_size);
  PK_REQUIRE(is_pow2(num_groups), "num_groups %zu is not a power of two", num_groups);
  PK_REQUIRE(len > 0 && len % codeword_size == 0,
             "len %zu is not a positive multiple of codeword_size %zu", len, codeword_size);
  PK_REQUIRE(codeword_size <= (size_t(1) << 28), "codeword_size %zu exceeds 2^28", codeword_size);
  if (num_groups >= codeword_size) *noop = 1;
  return PKG_OK;
}

int ntt_nr_device(uint64_t* values, size_t len, size_t codeword_size, size_t num_groups,
                  cudaStream_t stream) {
  int noop = 0;
  int rc = ntt_validate(len, codeword_size, num_groups, &noop);
  if (rc || noop) return rc;
  PK_REQUIRE(values != nullptr, "null values pointer");
  PK_REQUIRE(aligned16(values), "device buffers must be 16-byte aligned");
  const uint64_t* roots = nullptr;
  rc = roots_reserve(codeword_size, &roots);
  if (rc) return rc;
  size_t M = len / codeword_size;
  return ntt_stages(values, codeword_size, M, log2_exact(num_groups), log2_exact(codeword_size),
                    roots, stream);
}

int ntt_nr_from_source(uint64_t* out, size_t len, size_t codeword_size, size_t num_groups,
                       const NttSource& src, cudaStream_t stream) {
  int noop = 0;
  int rc = ntt_validate(len, codeword_size, num_groups, &noop);
  if (rc) return rc;
  PK_REQUIRE(!noop, "no transform stage to read the source");
  PK_REQUIRE(out != nullptr && aligned16(out), "null or unaligned output");
  const uint64_t* roots = nullptr;
  rc = roots_reserve(codeword_size, &roots);
  if (rc) return rc;
  return ntt_stages(out, codeword_size, len / codeword_size, log2_exact(num_groups),
                    log2_exact(codeword_size), roots, stream, &src);
}

// ---------------------------------------------------------------------------
// intt_rn: reverse_order -> values[1..].reverse() -> ntt_nr -> * n^-1 ->
// reverse_order (ntt/src/ntt.rs:326-348), as two gathers around the NTT:
//   v2[i] = v0[bitrev((n - i) mod n)]             (in -> tmp)
//   v4[i] = v3[bitrev(i)] * n^-1                   (tmp -> out)
// ---------------------------------------------------------------------------
__global__ void intt_gather_in(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                               size_t n, int log_n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    size_t k = (n - i) & (n - 1);
    size_t r = log_n ? (__brevll((unsigned long long)k) >> (64 - log_n)) : 0;
    fr_store(dst, i, fr_load(src, r));
  }
}

__global__ void intt_gather_out(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                size_t n, int log_n, Fr ninv) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    size_t r = log_n ? (__brevll((unsigned long long)i) >> (64 - log_n)) : 0;
    fr_store(dst, i, fr_mul(fr_load(src, r), ninv));
  }
}

int intt_rn_device(uint64_t* values, size_t len, cudaStream_t stream) {
  PK_REQUIRE(is_pow2(len), "intt_rn length %zu is not a power of two", len);
  PK_REQUIRE(len <= (size_t(1) << 28), "intt_rn length %zu exceeds 2^28", len);
  PK_REQUIRE(values != nullptr, "null values pointer");
  PK_REQUIRE(aligned16(values), "device buffers must be 16-byte aligned");
  if (len == 1) return PKG_OK;  // both permutations and the scale are identities
  Scratch tmp;
  int rc = tmp.alloc(32 * len, stream);
  if (rc) return rc;
  uint64_t* t = static_cast<uint64_t*>(tmp.ptr);
  int log_n = log2_exact(len);
  int blocks = (int)std::min<size_t>((len + 255) / 256, (size_t)sm_count() * 16);
  intt_gather_in<<<blocks, 256, 0, stream>>>(values, t, len, log_n);
  PK_CHECK_LAUNCH("intt_gather_in");
  rc = ntt_nr_device(t, len, len, 1, stream);
  if (rc) return rc;
  HostFr ninv = HostFr::inv(HostFr::from_u64(len));
  Fr nv;
  memcpy(nv.v, ninv.l, 32);
  intt_gather_out<<<blocks, 256, 0, stream>>>(t, values, len, log_n, nv);
  PK_CHECK_LAUNCH("intt_gather_out");
  return PKG_OK;
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_ntt_nr(uint64_t* values, size_t len, size_t codeword_size, size_t num_groups,
                          pkg_stream_t stream) {
  return ntt_nr_device(values, len, codeword_size, num_groups, as_stream(stream));
}

extern "C" int pkg_intt_rn(uint64_t* values, size_t len, pkg_stream_t stream) {
  return intt_rn_device(values, len, as_stream(stream));
}

extern "C" int pkg_ntt_engine_reserve(size_t order) {
  const uint64_t* r = nullptr;
  return roots_reserve(order, &r);
}

// In-place transform of a host slice through the host stager: one pipelined
// upload, the device transform on the stager's stream, one pipelined download.
static int host_transform(uint64_t* values, size_t len, size_t codeword_size,
                          size_t num_groups, bool inverse) {
  HostStager& hs = HostStager::current();
  std::lock_guard<std::mutex> lk(hs.mutex());
  uint8_t* ws = nullptr;
  int rc = hs.workspace(32 * len, &ws);
  if (rc) return rc;
  rc = hs.h2d(ws, values, 32 * len);
  if (rc) return rc;
  uint64_t* d = reinterpret_cast<uint64_t*>(ws);
  rc = inverse ? intt_rn_device(d, len, hs.stream())
               : ntt_nr_device(d, len, codeword_size, num_groups, hs.stream());
  if (rc) return rc;
  rc = hs.d2h(values, ws, 32 * len);
  if (rc) return rc;
  PK_CUDA(cudaStreamSynchronize(hs.stream()));
  return PKG_OK;
}

extern "C" int pkg_host_ntt_nr(uint64_t* values, size_t len, size_t codeword_size,
                               size_t num_groups) {
  int noop = 0;
  int rc = ntt_validate(len, codeword_size, num_groups, &noop);
  if (rc || noop) return rc;
  PK_REQUIRE(values != nullptr, "null values pointer");
  return host_transform(values, len, codeword_size, num_groups, false);
}

extern "C" int pkg_host_intt_rn(uint64_t* values, size_t len) {
  PK_REQUIRE(is_pow2(len), "intt_rn length %zu is not a power of two", len);
  PK_REQUIRE(values != nullptr, "null values pointer");
  return host_transform(values, len, len, 1, true);
}
