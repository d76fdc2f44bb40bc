// skyscraper.cu -- Skyscraper hashing and the Merkle commit on the device:
//   pkg_skyscraper_compress_many  simple::compress_many (skyscraper/core/src/simple.rs:3-9)
//   pkg_skyscraper_hash_many      SkyscraperHashEngine::hash_many
//                                 (provekit/common/src/skyscraper/whir.rs:42-100)
//   pkg_merkle_tree[_fr]          the binary tree WHIR builds from hash_many
//                                 (leaves: hash_many(leaf_size); nodes: hash_many(64))
//   pkg_skyscraper_pow_solve      generic::solve (skyscraper/core/src/generic.rs:42-71)
//   pkg_whir_commit               RS encode + Merkle tree of one polynomial
//
// One thread owns one compression chain (a leaf's left fold, or one node);
// 32-byte chunks are read as two 128-bit vector loads.  Levels above
// kSubtreeMax nodes take one launch each; below it one launch reduces
// 256-node subtrees per CTA by eight levels, and one CTA finishes the top in
// shared memory.
#include <algorithm>
#include <cstring>

#include "fr.cuh"
#include "ntt_internal.cuh"
#include "host_stage.cuh"
#include "internal.cuh"
#include "pk_common.cuh"
#include "rs_internal.cuh"
#include "skyscraper.cuh"

namespace pk {

constexpr int kTopNodes = 1024;  // nodes finished inside one CTA

// CTAs of 128 threads per SM the leaf kernel is compiled for (its register
// budget: 7 -> 72 registers).
#ifndef PK_LEAF_MIN_CTAS
#define PK_LEAF_MIN_CTAS 7
#endif

__device__ __forceinline__ Fr load_raw(const uint8_t* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 a = __ldg(q), b = __ldg(q + 1);
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}

__device__ __forceinline__ void store_raw(uint8_t* p, const Fr& x) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  q[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// ---- compress_many / hash_many -------------------------------------------
__global__ void compress_many_kernel(const uint8_t* __restrict__ in, size_t n,
                                     uint8_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr l = load_raw(in + 64 * i), r = load_raw(in + 64 * i + 32);
    store_raw(out + 32 * i, sky_compress(l, r));
  }
}

// Left fold h = c(c(c(e0, e1), e2), ...) over `chunks` 32-byte chunks
// (one compression call site keeps the register count low).
__global__ void leaf_fold_kernel(const uint8_t* __restrict__ in, size_t size, size_t chunks,
                                 size_t count, uint8_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint8_t* msg = in + i * size;
    Fr acc = load_raw(msg);
#pragma unroll 1
    for (size_t k = 1; k < chunks; k++) acc = sky_compress(acc, load_raw(msg + 32 * k));
    store_raw(out + 32 * i, acc);
  }
}

// Leaves straight from an Fr codeword: leaf i = row i (fr_per_leaf
// consecutive Fr).  Canonical encoding converts each Montgomery element
// (x*2^256 -> x) before hashing; Montgomery encoding hashes the raw limbs.
// A one-element leaf is the element itself (hash_many(32) copies).
template <bool kCanonical>
__global__ void __launch_bounds__(128, PK_LEAF_MIN_CTAS) leaf_fold_fr_kernel(const uint64_t* __restrict__ cw, size_t fr_per_leaf,
                                    size_t count, uint8_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t base = i * fr_per_leaf;
    Fr acc = fr_load_ro(cw, base);
    if (kCanonical) acc = fr_from_mont(acc);
#pragma unroll 1
    for (size_t k = 1; k < fr_per_leaf; k++) {
      Fr e = fr_load_ro(cw, base + k);
      if (kCanonical) e = fr_from_mont(e);
      acc = sky_compress(acc, e);
    }
    store_raw(out + 32 * i, acc);
  }
}

// One tree level: out[i] = compress(in[2i], in[2i+1]).
__global__ void merkle_level_kernel(const uint8_t* __restrict__ in, size_t n_out,
                                    uint8_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_out;
       i += (size_t)gridDim.x * blockDim.x) {
    store_raw(out + 32 * i, sky_compress(load_raw(in + 64 * i), load_raw(in + 64 * i + 32)));
  }
}

// The remaining levels from n (<= kTopNodes, power of two) nodes up to the
// root, in one CTA: level digests live in shared memory and are also written
// out to their slots in the layer array.
__global__ void __launch_bounds__(512) merkle_top_kernel(const uint8_t* __restrict__ in,
                                                         size_t n, uint8_t* __restrict__ out) {
  __shared__ uint4 buf[2 * kTopNodes];
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint4* q = reinterpret_cast<const uint4*>(in + 32 * i);
    buf[2 * i] = q[0];
    buf[2 * i + 1] = q[1];
  }
  __syncthreads();
  size_t off = 0;
  while (n > 1) {
    const size_t half = n / 2;  // <= blockDim.x: one node per thread
    Fr h;
    if (threadIdx.x < half) {
      const size_t i = threadIdx.x;
      Fr l, r;
      uint4 a = buf[4 * i], b = buf[4 * i + 1], c = buf[4 * i + 2], d = buf[4 * i + 3];
      l.v[0] = a.x; l.v[1] = a.y; l.v[2] = a.z; l.v[3] = a.w;
      l.v[4] = b.x; l.v[5] = b.y; l.v[6] = b.z; l.v[7] = b.w;
      r.v[0] = c.x; r.v[1] = c.y; r.v[2] = c.z; r.v[3] = c.w;
      r.v[4] = d.x; r.v[5] = d.y; r.v[6] = d.z; r.v[7] = d.w;
      h = sky_compress(l, r);
    }
    __syncthreads();
    if (threadIdx.x < half) {
      const size_t i = threadIdx.x;
      buf[2 * i] = make_uint4(h.v[0], h.v[1], h.v[2], h.v[3]);
      buf[2 * i + 1] = make_uint4(h.v[4], h.v[5], h.v[6], h.v[7]);
      store_raw(out + 32 * (off + i), h);
    }
    __syncthreads();
    off += half;
    n = half;
  }
}

// The levels from kSubtreeMax nodes down: each CTA (one warp per SM
// sub-partition) reduces kSubNodes consecutive nodes of the current level by
// kSubLevels levels in shared memory and writes every level's digests to
// their slots, so the latency-bound small levels cost one launch instead of
// one each; the kSubNodes-fold fewer subroots go to merkle_top_kernel.
constexpr int kSubThreads = 128;
constexpr int kSubNodes = 2 * kSubThreads;
constexpr int kSubLevels = 8;  // kSubNodes = 2^kSubLevels
constexpr size_t kSubtreeMax = size_t(1) << 15;
static_assert(kSubNodes == 1 << kSubLevels, "a CTA reduces its nodes to one subroot");
static_assert(kSubtreeMax / kSubNodes <= (size_t)kTopNodes, "the subroots fit the top kernel");

__global__ void __launch_bounds__(kSubThreads) merkle_subtree_kernel(uint8_t* __restrict__ lvl,
                                                                     size_t n) {
  __shared__ uint4 buf[2 * kSubNodes];
  const size_t c = blockIdx.x;  // this CTA's nodes: [c kSubNodes, (c + 1) kSubNodes)
  for (int i = threadIdx.x; i < kSubNodes; i += blockDim.x) {
    const uint4* q = reinterpret_cast<const uint4*>(lvl + 32 * (c * kSubNodes + i));
    buf[2 * i] = q[0];
    buf[2 * i + 1] = q[1];
  }
  __syncthreads();
  uint8_t* level = lvl;  // first node of the current level
  size_t level_n = n;
  int cnt = kSubNodes;
#pragma unroll 1
  for (int l = 0; l < kSubLevels; l++) {
    const int half = cnt / 2;
    const int i = threadIdx.x;
    Fr h;
    if (i < half) {
      Fr a, b;
      const uint4 x0 = buf[4 * i], x1 = buf[4 * i + 1], y0 = buf[4 * i + 2], y1 = buf[4 * i + 3];
      a.v[0] = x0.x; a.v[1] = x0.y; a.v[2] = x0.z; a.v[3] = x0.w;
      a.v[4] = x1.x; a.v[5] = x1.y; a.v[6] = x1.z; a.v[7] = x1.w;
      b.v[0] = y0.x; b.v[1] = y0.y; b.v[2] = y0.z; b.v[3] = y0.w;
      b.v[4] = y1.x; b.v[5] = y1.y; b.v[6] = y1.z; b.v[7] = y1.w;
      h = sky_compress(a, b);
    }
    __syncthreads();
    uint8_t* next = level + 32 * level_n;
    if (i < half) {
      buf[2 * i] = make_uint4(h.v[0], h.v[1], h.v[2], h.v[3]);
      buf[2 * i + 1] = make_uint4(h.v[4], h.v[5], h.v[6], h.v[7]);
      store_raw(next + 32 * (c * half + i), h);
    }
    __syncthreads();
    level = next;
    level_n /= 2;
    cnt = half;
  }
}

static int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  size_t cap = (size_t)sm_count() * 64;
  return (int)std::max<size_t>(1, std::min(b, cap));
}

int compress_many_device(const uint8_t* in, size_t n, uint8_t* out, cudaStream_t s) {
  if (n == 0) return PKG_OK;
  PK_REQUIRE(in && out, "null pointer");
  PK_REQUIRE(aligned16(in) && aligned16(out), "device buffers must be 16-byte aligned");
  compress_many_kernel<<<grid_for(n, 128), 128, 0, s>>>(in, n, out);
  PK_CHECK_LAUNCH("compress_many_kernel");
  return PKG_OK;
}

int hash_many_device(size_t size, const uint8_t* in, size_t count, uint8_t* out, cudaStream_t s) {
  PK_REQUIRE(size > 0 && size % 32 == 0,
             "skyscraper: unsupported message size %zu (must be a positive multiple of 32)",
             size);
  if (count == 0) return PKG_OK;
  PK_REQUIRE(in && out, "null pointer");
  PK_REQUIRE(aligned16(in) && aligned16(out), "device buffers must be 16-byte aligned");
  if (size == 32) {
    PK_CUDA(cudaMemcpyAsync(out, in, 32 * count, cudaMemcpyDeviceToDevice, s));
    return PKG_OK;
  }
  if (size == 64) return compress_many_device(in, count, out, s);
  leaf_fold_kernel<<<grid_for(count, 128), 128, 0, s>>>(in, size, size / 32, count, out);
  PK_CHECK_LAUNCH("leaf_fold_kernel");
  return PKG_OK;
}

// Internal levels above the leaf digests already in layers[0..n) (n a power
// of two): one launch per level while a level has more than kSubtreeMax
// nodes, then the subtree kernel's kSubLevels levels, then the top.
int merkle_levels_device(uint8_t* layers, size_t n, cudaStream_t s) {
  uint8_t* cur = layers;
  while (n > kSubtreeMax) {
    uint8_t* next = cur + 32 * n;
    merkle_level_kernel<<<grid_for(n / 2, 128), 128, 0, s>>>(cur, n / 2, next);
    PK_CHECK_LAUNCH("merkle_level_kernel");
    cur = next;
    n /= 2;
  }
  if (n >= (size_t)kSubNodes * 2) {
    merkle_subtree_kernel<<<(unsigned)(n / kSubNodes), kSubThreads, 0, s>>>(cur, n);
    PK_CHECK_LAUNCH("merkle_subtree_kernel");
    for (int l = 0; l < kSubLevels; l++) {
      cur += 32 * n;
      n /= 2;
    }
  }
  if (n > 1) {
    merkle_top_kernel<<<1, 512, 0, s>>>(cur, n, cur + 32 * n);
    PK_CHECK_LAUNCH("merkle_top_kernel");
  }
  return PKG_OK;
}

int merkle_leaves_fr_device(const uint64_t* cw, size_t fr_per_leaf, size_t num_leaves,
                            int encoding, uint8_t* layers, cudaStream_t s) {
  PK_REQUIRE(is_pow2(num_leaves), "num_leaves %zu is not a power of two", num_leaves);
  PK_REQUIRE(fr_per_leaf >= 1, "fr_per_leaf must be >= 1");
  PK_REQUIRE(encoding == PKG_LEAF_CANONICAL || encoding == PKG_LEAF_MONTGOMERY,
             "unknown leaf encoding %d", encoding);
  PK_REQUIRE(cw && layers, "null pointer");
  PK_REQUIRE(aligned16(cw) && aligned16(layers), "device buffers must be 16-byte aligned");
  int g = grid_for(num_leaves, 128);
  if (encoding == PKG_LEAF_CANONICAL)
    leaf_fold_fr_kernel<true><<<g, 128, 0, s>>>(cw, fr_per_leaf, num_leaves, layers);
  else
    leaf_fold_fr_kernel<false><<<g, 128, 0, s>>>(cw, fr_per_leaf, num_leaves, layers);
  PK_CHECK_LAUNCH("leaf_fold_fr_kernel");
  return PKG_OK;
}

int merkle_tree_fr_device(const uint64_t* cw, size_t fr_per_leaf, size_t num_leaves,
                          int encoding, uint8_t* layers, cudaStream_t s) {
  int rc = merkle_leaves_fr_device(cw, fr_per_leaf, num_leaves, encoding, layers, s);
  if (rc) return rc;
  return merkle_levels_device(layers, num_leaves, s);
}

// ---- PoW -----------------------------------------------------------------
__global__ void pow_kernel(Fr challenge, Fr threshold, uint64_t base, uint64_t n,
                           unsigned long long* best) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t nonce = base + i;
    Fr r = fr_zero();
    r.v[0] = (uint32_t)nonce;
    r.v[1] = (uint32_t)(nonce >> 32);
    Fr h = sky_compress(challenge, r);
    bool lt = false;
#pragma unroll
    for (int k = 7; k >= 0; k--) {  // less_than, arithmetic.rs:447-456
      if (h.v[k] != threshold.v[k]) {
        lt = h.v[k] < threshold.v[k];
        break;
      }
    }
    if (lt) atomicMin(best, (unsigned long long)nonce);
  }
}

// The smallest nonce with compress(challenge, [nonce,0,0,0]) < threshold:
// batches of candidates in increasing order, starting small (a PoW of b
// bits needs about 2^b candidates) and growing four-fold, so the first
// batch that holds a solution holds the smallest one.
int pow_solve_device(const uint64_t challenge[4], const uint64_t threshold[4], cudaStream_t s,
                     uint64_t* nonce_out) {
  Fr c, t;
  memcpy(c.v, challenge, 32);
  memcpy(t.v, threshold, 32);
  bool thr_zero = true;
  for (int i = 0; i < 8; i++) thr_zero &= (t.v[i] == 0);
  PK_REQUIRE(!thr_zero, "threshold 0 admits no nonce");
  // the best nonce in the thread's own PoW word (after the fused
  // reductions' partials, which it never overlaps): no pool allocation per PoW
  FusedSlots fs;
  int rc = fused_slots(&fs);
  if (rc) return rc;
  unsigned long long* d_best = fs.pow;
  PK_CUDA(cudaMemsetAsync(d_best, 0xff, sizeof(unsigned long long), s));
  const unsigned long long none = ~0ULL;
  unsigned long long best = none;
  const uint64_t max_batch = uint64_t(1) << 22;
  uint64_t batch = uint64_t(1) << 13;
  for (uint64_t base = 0; best == none; base += batch, batch = std::min(batch * 4, max_batch)) {
    if (base > (uint64_t(1) << 62)) break;
    const int grid = (int)std::min<uint64_t>((uint64_t)sm_count() * 8, (batch + 255) / 256);
    pow_kernel<<<grid, 256, 0, s>>>(c, t, base, batch, d_best);
    PK_CHECK_LAUNCH("pow_kernel");
    if ((rc = read_small(&best, d_best, sizeof best, s))) return rc;
  }
  if (best == none) {
    set_last_error("no nonce found");
    return PKG_ERR_UNSUPPORTED;
  }
  *nonce_out = best;
  return PKG_OK;
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_skyscraper_compress_many(const uint8_t* messages, size_t count,
                                            uint8_t* hashes, pkg_stream_t stream) {
  return compress_many_device(messages, count, hashes, as_stream(stream));
}

extern "C" int pkg_skyscraper_hash_many(size_t size, const uint8_t* input, size_t count,
                                        uint8_t* output, pkg_stream_t stream) {
  return hash_many_device(size, input, count, output, as_stream(stream));
}

extern "C" int pkg_host_skyscraper_hash_many(size_t size, const uint8_t* input, size_t count,
                                             uint8_t* output) {
  PK_REQUIRE(size > 0 && size % 32 == 0,
             "skyscraper: unsupported message size %zu (must be a positive multiple of 32)",
             size);
  if (count == 0) return PKG_OK;
  PK_REQUIRE(input && output, "null pointer");
  const size_t in_span = (size * count + 255) & ~size_t(255);
  HostStager& hs = HostStager::current();
  std::lock_guard<std::mutex> lk(hs.mutex());
  uint8_t* ws = nullptr;
  int rc = hs.workspace(in_span + 32 * count, &ws);
  if (rc) return rc;
  rc = hs.h2d(ws, input, size * count);
  if (rc) return rc;
  rc = hash_many_device(size, ws, count, ws + in_span, hs.stream());
  if (rc) return rc;
  rc = hs.d2h(output, ws + in_span, 32 * count);
  if (rc) return rc;
  PK_CUDA(cudaStreamSynchronize(hs.stream()));
  return PKG_OK;
}

extern "C" int pkg_merkle_tree(const uint8_t* leaves, size_t leaf_size, size_t num_leaves,
                               uint8_t* layers, pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(num_leaves), "num_leaves %zu is not a power of two", num_leaves);
  cudaStream_t s = as_stream(stream);
  int rc = hash_many_device(leaf_size, leaves, num_leaves, layers, s);
  if (rc) return rc;
  return merkle_levels_device(layers, num_leaves, s);
}

extern "C" int pkg_merkle_tree_fr(const uint64_t* codeword, size_t fr_per_leaf,
                                  size_t num_leaves, int leaf_encoding, uint8_t* layers,
                                  pkg_stream_t stream) {
  return merkle_tree_fr_device(codeword, fr_per_leaf, num_leaves, leaf_encoding, layers,
                               as_stream(stream));
}

extern "C" int pkg_merkle_leaves_fr(const uint64_t* codeword, size_t fr_per_leaf,
                                    size_t num_leaves, int leaf_encoding, uint8_t* layers,
                                    pkg_stream_t stream) {
  return merkle_leaves_fr_device(codeword, fr_per_leaf, num_leaves, leaf_encoding, layers,
                                 as_stream(stream));
}

extern "C" int pkg_merkle_levels(uint8_t* layers, size_t num_leaves, pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(num_leaves), "num_leaves %zu is not a power of two", num_leaves);
  PK_REQUIRE(layers && aligned16(layers), "layers must be a 16-byte aligned device pointer");
  return merkle_levels_device(layers, num_leaves, as_stream(stream));
}

extern "C" int pkg_whir_commit(const uint64_t* coeffs, size_t num_coeffs,
                               unsigned folding_factor, unsigned log_inv_rate,
                               const uint64_t* masks, size_t mask_len, int leaf_encoding,
                               uint64_t* codeword_out, uint8_t* layers_out,
                               pkg_stream_t stream) {
  PK_REQUIRE(folding_factor <= 12 && log_inv_rate <= 28, "unsupported folding factor / rate");
  size_t M = size_t(1) << folding_factor;
  PK_REQUIRE(is_pow2(num_coeffs) && num_coeffs >= M,
             "num_coeffs %zu must be a power of two >= 2^folding_factor", num_coeffs);
  size_t L = num_coeffs / M;
  PK_REQUIRE((L << log_inv_rate) <= (size_t(1) << 28),
             "codeword of %zu << %u rows exceeds the largest NTT order 2^28", L, log_inv_rate);
  size_t cw_len = L << log_inv_rate;
  cudaStream_t s = as_stream(stream);
  int rc = rs_encode_device(coeffs, M, L, masks, mask_len, cw_len, codeword_out, s);
  if (rc) return rc;
  return merkle_tree_fr_device(codeword_out, M, cw_len, leaf_encoding, layers_out, s);
}

extern "C" int pkg_skyscraper_pow_solve(const uint64_t challenge[4], const uint64_t threshold[4],
                                        uint64_t* nonce_out) {
  PK_REQUIRE(challenge && threshold && nonce_out, "null pointer");
  cudaStream_t s = nullptr;
  PK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int rc = pow_solve_device(challenge, threshold, s, nonce_out);
  cudaStreamDestroy(s);
  return rc;
}
