// noalloc.cu -- pkg_intt_rn_noalloc: the inverse NTT without any device
// allocation.
//
// pkg_intt_rn needs scratch memory (a gather buffer of len Fr from
// cudaMallocAsync, plus the twiddle table, which grows with cudaMalloc).
// Some callers cannot let a library allocate device memory: a prover service
// that reserves all HBM up front for its own admission control, or a host
// application whose framework allocator owns every free byte; cudaMalloc and
// cudaFree can also synchronise the device, which latency-critical loops
// avoid.  This variant keeps its scratch in one file-scope __device__ array
// of fixed size instead: every GPU that loads the library holds
// kNoAllocScratchBytes (3 MiB) of it until the process exits.
//
// Host code must not use the array's name as a device address (in host code
// it is only a stand-in symbol).  The first call on each device looks the
// address up with cudaGetSymbolAddress while that device is current and
// caches it; make that first call before capturing any stream.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "fr.cuh"
#include "fr_host.hpp"
#include "ntt_internal.cuh"
#include "pk_common.cuh"

namespace pk {

constexpr size_t kNoAllocMaxLen = size_t(1) << 16;
// twiddles (len/2 Fr) followed by the gather buffer (len Fr)
constexpr size_t kNoAllocScratchFr = kNoAllocMaxLen / 2 + kNoAllocMaxLen;
constexpr size_t kNoAllocScratchBytes = 32 * kNoAllocScratchFr;
static_assert(kNoAllocScratchBytes == (size_t(3) << 20), "3 MiB of fixed scratch");

static __device__ __align__(256) uint64_t g_noalloc_scratch[4 * kNoAllocScratchFr];

static std::mutex g_noalloc_mu;
static std::vector<uint64_t*> g_noalloc_ptr;  // per device, from cudaGetSymbolAddress

static int noalloc_scratch(uint64_t** out) {
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if ((int)g_noalloc_ptr.size() <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[dev] = static_cast<uint64_t*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return PKG_OK;
}

// roots[bitrev(i)] = w^i for i < n/2 (square-and-multiply per entry; the
// values equal the shared table's, entry by entry).
__global__ void noalloc_roots_kernel(uint64_t* __restrict__ roots, size_t half, int log_half,
                                     Fr w) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half;
       i += (size_t)gridDim.x * blockDim.x) {
    Fr acc = fr_one_mont(), base = w;
    for (size_t e = i; e; e >>= 1) {
      if (e & 1) acc = fr_mul(acc, base);
      base = fr_sqr(base);
    }
    size_t r = log_half ? (__brevll((unsigned long long)i) >> (64 - log_half)) : 0;
    fr_store(roots, r, acc);
  }
}

// dst[i] = src[bitrev((n - i) mod n)]
__global__ void noalloc_gather_in(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                  size_t n, int log_n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    size_t k = (n - i) & (n - 1);
    size_t r = __brevll((unsigned long long)k) >> (64 - log_n);
    fr_store(dst, i, fr_load(src, r));
  }
}

// dst[i] = src[bitrev(i)] * n^-1
__global__ void noalloc_gather_out(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                   size_t n, int log_n, Fr ninv) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    size_t r = __brevll((unsigned long long)i) >> (64 - log_n);
    fr_store(dst, i, fr_mul(fr_load(src, r), ninv));
  }
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_intt_rn_noalloc(uint64_t* values, size_t len, pkg_stream_t stream) {
  PK_REQUIRE(is_pow2(len), "intt_rn length %zu is not a power of two", len);
  PK_REQUIRE(len <= kNoAllocMaxLen,
             "pkg_intt_rn_noalloc: length %zu exceeds the fixed scratch maximum %zu", len,
             kNoAllocMaxLen);
  PK_REQUIRE(values != nullptr && aligned16(values),
             "values must be a 16-byte aligned device pointer");
  if (len == 1) return PKG_OK;  // both permutations and the scale are identities
  uint64_t* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  const int log_n = log2_exact(len);
  uint64_t* roots = scratch;                     // len/2 Fr
  uint64_t* tmp = scratch + 4 * (kNoAllocMaxLen / 2);  // len Fr
  // Every scratch word this call reads is written by this call first.
  HostFr w = HostFr::root_of_unity(len);
  Fr wd;
  memcpy(wd.v, w.l, 32);
  const int blocks = (int)std::min<size_t>((len + 255) / 256, (size_t)sm_count() * 8);
  noalloc_roots_kernel<<<blocks, 256, 0, s>>>(roots, len / 2, log_n - 1, wd);
  PK_CHECK_LAUNCH("noalloc_roots_kernel");
  noalloc_gather_in<<<blocks, 256, 0, s>>>(values, tmp, len, log_n);
  PK_CHECK_LAUNCH("noalloc_gather_in");
  rc = ntt_stages(tmp, len, 1, 0, log_n, roots, s);
  if (rc) return rc;
  HostFr ninv = HostFr::inv(HostFr::from_u64(len));
  Fr nv;
  memcpy(nv.v, ninv.l, 32);
  noalloc_gather_out<<<blocks, 256, 0, s>>>(tmp, values, len, log_n, nv);
  PK_CHECK_LAUNCH("noalloc_gather_out");
  return PKG_OK;
}
