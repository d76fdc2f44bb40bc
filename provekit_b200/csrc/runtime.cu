// runtime.cu -- library-wide plumbing: last-error storage, version, device
// properties, the host-side Fr sampler and the IMAD-rate microbenchmark.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "fr_host.hpp"
#include "pk_common.cuh"

namespace pk {

static thread_local char g_last_error[512] = "";

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
  va_end(ap);
}

void clear_last_error() { g_last_error[0] = 0; }

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches_undo(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }

int sm_count() {
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
  if (!cache[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n > 0 ? n : 148;
  }
  return cache[dev];
}

// ---------------------------------------------------------------------------
// ChaCha20 sampler (RFC 8439 section 2.3 block function).
// ---------------------------------------------------------------------------
static inline uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

static void chacha20_block(const uint32_t key[8], uint64_t counter, uint32_t out[16]) {
  const uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                          key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                          (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u};
  uint32_t x[16];
  memcpy(x, s, sizeof x);
  auto qr = [&](int a, int b, int c, int d) {
    x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 16);
    x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 12);
    x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 8);
    x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 7);
  };
  for (int i = 0; i < 10; i++) {
    qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
    qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// ---------------------------------------------------------------------------
// IMAD microbenchmark: 8 independent mad.lo.cc/madc.hi.cc chains per thread.
// ---------------------------------------------------------------------------
__global__ void imad_rate_kernel(uint32_t* sink, uint32_t seed, int iters) {
  uint32_t a0 = seed ^ threadIdx.x, a1 = a0 * 3u + 1u, a2 = a1 * 5u + 7u, a3 = a2 * 9u + 3u;
  uint32_t b = seed * 0x9e3779b9u + blockIdx.x;
  uint32_t c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0, c7 = 0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      asm volatile(
          "mad.lo.cc.u32  %0, %8,  %12, %0;\n\t"
          "madc.hi.cc.u32 %1, %8,  %12, %1;\n\t"
          "madc.lo.cc.u32 %2, %9,  %12, %2;\n\t"
          "madc.hi.cc.u32 %3, %9,  %12, %3;\n\t"
          "madc.lo.cc.u32 %4, %10, %12, %4;\n\t"
          "madc.hi.cc.u32 %5, %10, %12, %5;\n\t"
          "madc.lo.cc.u32 %6, %11, %12, %6;\n\t"
          "madc.hi.u32    %7, %11, %12, %7;"
          : "+r"(c0), "+r"(c1), "+r"(c2), "+r"(c3), "+r"(c4), "+r"(c5), "+r"(c6), "+r"(c7)
          : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b));
    }
  }
  uint32_t s = c0 ^ c1 ^ c2 ^ c3 ^ c4 ^ c5 ^ c6 ^ c7;
  if (s == 0x12345678u) sink[threadIdx.x] = s;
}

// Eight independent fma chains per thread; x -> x * c + d converges to
// d / (1 - c) and never leaves the normal range.
__global__ void dfma_rate_kernel(double* sink, double c, double d, int iters) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
         x6 = x0 + 6, x7 = x0 + 7;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      x0 = fma(x0, c, d); x1 = fma(x1, c, d); x2 = fma(x2, c, d); x3 = fma(x3, c, d);
      x4 = fma(x4, c, d); x5 = fma(x5, c, d); x6 = fma(x6, c, d); x7 = fma(x7, c, d);
    }
  }
  const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == -1.0) sink[threadIdx.x] = s;
}

// ---------------------------------------------------------------------------
// Per-thread resources, owned by one thread_local object and released when
// the thread exits (or by pkg_release_thread_resources).
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kBounceCap = size_t(256) << 10;
// the fused slots, then the completion word fused launches write (64 bytes)
constexpr size_t kFusedHostBytes = 32 * kFusedSlotFr + 64;
std::atomic<int64_t> g_res_host{0}, g_res_dev{0};

// the device block of one thread on one device: the ticket counter, the
// partials of one reduction launch (3 Fr for each of 4 CTAs per SM), then the
// PoW search's word
size_t fused_block_bytes() { return 256 + 32 * 3 * 4 * (size_t)sm_count() + 256; }

struct ThreadResources {
  uint64_t* fused_host = nullptr;  // mapped pinned, portable
  uint64_t* fused_dev = nullptr;
  struct PerDevice {
    uint8_t* block = nullptr;  // ticket, partials, PoW word
    size_t block_bytes = 0;
    unsigned seq = 0;          // the last completion number handed out
    PinnedStage stage;
  };
  PerDevice dev[kMaxDevices];
  uint8_t* bounce = nullptr;
  bool bounce_tried = false;
#ifdef PK_DEBUG_FUSED
  bool fused_busy = false;
#endif

  void release() {
    int cur = -1;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    for (int d = 0; d < kMaxDevices; d++) {
      PerDevice& pd = dev[d];
      if (!pd.block && !pd.stage.buf && !pd.stage.copied) continue;
      cudaSetDevice(d);
      // copies into the stage may still be in flight: wait for the last one
      if (pd.stage.copied) {
        cudaEventSynchronize(pd.stage.copied);
        cudaEventDestroy(pd.stage.copied);
      }
      if (pd.stage.buf) {
        cudaFreeHost(pd.stage.buf);
        g_res_host -= (int64_t)pd.stage.cap;
      }
      if (pd.block) {
        cudaFree(pd.block);  // waits for the device's outstanding work
        g_res_dev -= (int64_t)pd.block_bytes;
      }
      pd = PerDevice();
    }
    if (have_cur) cudaSetDevice(cur);
    if (fused_host) {
      cudaFreeHost(fused_host);
      g_res_host -= (int64_t)kFusedHostBytes;
    }
    if (bounce) {
      cudaFreeHost(bounce);
      g_res_host -= (int64_t)kBounceCap;
    }
    fused_host = fused_dev = nullptr;
    bounce = nullptr;
    bounce_tried = false;
    cudaGetLastError();  // a teardown-time failure is not the caller's error
  }
  ~ThreadResources() { release(); }
};

thread_local ThreadResources t_res;

}  // namespace

void thread_resource_totals(size_t* host_bytes, size_t* device_bytes) {
  *host_bytes = (size_t)std::max<int64_t>(0, g_res_host.load());
  *device_bytes = (size_t)std::max<int64_t>(0, g_res_dev.load());
}

// The thread's mapped pinned buffer: the fused slots, the completion word
// (byte 32 kFusedSlotFr) and the spare word (16 bytes later).
static int fused_host_buffer(ThreadResources& tr) {
  if (tr.fused_host) return PKG_OK;
  void* p = nullptr;
  PK_CUDA(cudaHostAlloc(&p, kFusedHostBytes, cudaHostAllocMapped | cudaHostAllocPortable));
  memset(p, 0, kFusedHostBytes);
  void* d = nullptr;
  const cudaError_t e = cudaHostGetDevicePointer(&d, p, 0);
  if (e != cudaSuccess) {
    cudaFreeHost(p);
    return cuda_status(e, "cudaHostGetDevicePointer");
  }
  tr.fused_host = static_cast<uint64_t*>(p);
  tr.fused_dev = static_cast<uint64_t*>(d);
  g_res_host += (int64_t)kFusedHostBytes;
  return PKG_OK;
}

int fused_aux_word(uint32_t** word) {
  ThreadResources& tr = t_res;
  const int rc = fused_host_buffer(tr);
  if (rc) return rc;
  *word = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(tr.fused_host) +
                                      32 * kFusedSlotFr + 16);
  return PKG_OK;
}

int fused_slots(FusedSlots* f) {
  ThreadResources& tr = t_res;
#ifdef PK_DEBUG_FUSED
  PK_REQUIRE(!tr.fused_busy,
             "fused slots: a fused use began before the thread's previous one synchronised");
  tr.fused_busy = true;
#endif
  {
    const int rc = fused_host_buffer(tr);
    if (rc) return rc;
  }
  int device = 0;
  PK_CUDA(cudaGetDevice(&device));
  PK_REQUIRE(device >= 0 && device < kMaxDevices, "device ordinal %d out of range", device);
  ThreadResources::PerDevice& pd = tr.dev[device];
  if (!pd.block) {
    // the counter and, 8 bytes in, the device address of the completion word
    // (written on a private stream, waited for: ordered before any later
    // launch on any stream without touching the legacy default stream),
    // followed by the partials of one reduction launch and the PoW word
    const size_t bytes = fused_block_bytes();
    void* t = nullptr;
    PK_CUDA(cudaMalloc(&t, bytes));
    unsigned* word_dev = reinterpret_cast<unsigned*>(
        reinterpret_cast<uint8_t*>(tr.fused_dev) + 32 * kFusedSlotFr);
    cudaStream_t z = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&z, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      e = cudaMemsetAsync(t, 0, 256, z);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(static_cast<uint8_t*>(t) + 8, &word_dev, sizeof word_dev,
                            cudaMemcpyHostToDevice, z);
      const cudaError_t e2 = cudaStreamSynchronize(z);
      if (e == cudaSuccess) e = e2;
      cudaStreamDestroy(z);
    }
    if (e != cudaSuccess) {
      cudaFree(t);
      return cuda_status(e, "fused slots: zeroing the ticket");
    }
    pd.block = static_cast<uint8_t*>(t);
    pd.block_bytes = bytes;
    g_res_dev += (int64_t)bytes;
  }
  f->host = tr.fused_host;
  f->dev = tr.fused_dev;
  f->ticket = reinterpret_cast<unsigned*>(pd.block);
  f->part = reinterpret_cast<uint64_t*>(pd.block + 256);
  f->pow = reinterpret_cast<unsigned long long*>(pd.block + pd.block_bytes - 256);
  return PKG_OK;
}

unsigned fused_next_seq() {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return 0;
  ThreadResources::PerDevice& pd = t_res.dev[device];
  if (++pd.seq == 0) pd.seq = 1;  // 0 means "no completion word"
  return pd.seq;
}

int fused_read(void* dst, const FusedSlots& f, size_t bytes, cudaStream_t s) {
  PK_REQUIRE(bytes <= 32 * kFusedSlotFr, "%zu bytes exceed the fused slots", bytes);
  int device = 0;
  PK_CUDA(cudaGetDevice(&device));
  const unsigned want = device >= 0 && device < kMaxDevices ? t_res.dev[device].seq : 0;
  volatile const unsigned* word =
      reinterpret_cast<volatile const unsigned*>(reinterpret_cast<const uint8_t*>(f.host) +
                                                 32 * kFusedSlotFr);
  // Poll the completion word the last fused launch writes after its sums
  // (a few microseconds sooner than the stream's own completion); the
  // stream's state is checked now and then, so an error, or a stream that
  // went idle without the word (a launch that wrote none), ends the poll and
  // falls back to synchronising.
  bool seen = false;
  for (uint32_t i = 1; want != 0; i++) {
    if (*word == want) {
      seen = true;
      break;
    }
    if ((i & 255) == 0) {
      const cudaError_t q = cudaStreamQuery(s);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_status(q, "fused_read");
    }
  }
  if (!seen) PK_CUDA(cudaStreamSynchronize(s));
#ifdef PK_DEBUG_FUSED
  t_res.fused_busy = false;
#endif
  memcpy(dst, f.host, bytes);
  return PKG_OK;
}

int pinned_stage(size_t bytes, PinnedStage** out) {
  int device = 0;
  PK_CUDA(cudaGetDevice(&device));
  PK_REQUIRE(device >= 0 && device < kMaxDevices, "device ordinal %d out of range", device);
  PinnedStage& st = t_res.dev[device].stage;
  if (!st.copied) PK_CUDA(cudaEventCreateWithFlags(&st.copied, cudaEventDisableTiming));
  PK_CUDA(cudaEventSynchronize(st.copied));
  if (bytes > st.cap) {
    if (st.buf) {
      cudaFreeHost(st.buf);
      g_res_host -= (int64_t)st.cap;
    }
    st.buf = nullptr;
    st.cap = 0;
    void* p = nullptr;
    PK_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocPortable));
    st.buf = static_cast<uint8_t*>(p);
    st.cap = bytes;
    g_res_host += (int64_t)bytes;
  }
  *out = &st;
  return PKG_OK;
}

// The bounce buffer of read_small, allocated on the thread's first use; a
// thread that cannot get one copies directly.
static void ensure_bounce(ThreadResources& tr) {
  if (tr.bounce_tried) return;
  tr.bounce_tried = true;
  void* p = nullptr;
  if (cudaHostAlloc(&p, kBounceCap, cudaHostAllocPortable) == cudaSuccess) {
    tr.bounce = static_cast<uint8_t*>(p);
    g_res_host += (int64_t)kBounceCap;
  } else {
    cudaGetLastError();  // no bounce buffer: direct copies
  }
}

int warm_thread_resources(size_t stage_bytes) {
  FusedSlots f;
  int rc = fused_slots(&f);
  if (rc) return rc;
#ifdef PK_DEBUG_FUSED
  t_res.fused_busy = false;
#endif
  ensure_bounce(t_res);
  PinnedStage* st = nullptr;
  return pinned_stage(stage_bytes, &st);
}

int read_small(const HostRead* reads, int n, cudaStream_t s) {
  ThreadResources& tr = t_res;
  ensure_bounce(tr);
  size_t total = 0;
  for (int i = 0; i < n; i++) total += (reads[i].bytes + 15) & ~size_t(15);
  if (!tr.bounce || total > kBounceCap) {
    for (int i = 0; i < n; i++)
      PK_CUDA(cudaMemcpyAsync(reads[i].dst, reads[i].src, reads[i].bytes, cudaMemcpyDeviceToHost,
                              s));
    PK_CUDA(cudaStreamSynchronize(s));
#ifdef PK_DEBUG_FUSED
    tr.fused_busy = false;
#endif
    return PKG_OK;
  }
  size_t off = 0;
  for (int i = 0; i < n; i++) {
    PK_CUDA(cudaMemcpyAsync(tr.bounce + off, reads[i].src, reads[i].bytes, cudaMemcpyDeviceToHost,
                            s));
    off += (reads[i].bytes + 15) & ~size_t(15);
  }
  PK_CUDA(cudaStreamSynchronize(s));
#ifdef PK_DEBUG_FUSED
  tr.fused_busy = false;
#endif
  off = 0;
  for (int i = 0; i < n; i++) {
    memcpy(reads[i].dst, tr.bounce + off, reads[i].bytes);
    off += (reads[i].bytes + 15) & ~size_t(15);
  }
  return PKG_OK;
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaMemPool_t lib_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    // A block freed on one stream is handed to another only once its free
    // has completed, never with a dependency the driver inserts between the
    // two streams: proofs running concurrently on their own streams would
    // otherwise be chained to each other's frees.  The pool grows instead.
    int no = 0;
    cudaMemPoolSetAttribute(p, cudaMemPoolReuseAllowInternalDependencies, &no);
    g_pools[dev] = p;
  }
  return g_pools[dev];
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_reserve_memory(size_t bytes) {
  cudaMemPool_t p = lib_pool();
  if (!p) {
    set_last_error("could not create the library memory pool");
    return PKG_ERR_CUDA;
  }
  if (bytes == 0) return PKG_OK;
  cudaStream_t ps = nullptr;
  PK_CUDA(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
  void* blk = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&blk, bytes, p, ps);
  if (e == cudaSuccess) e = cudaFreeAsync(blk, ps);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ps);
  cudaStreamDestroy(ps);
  if (e != cudaSuccess) return cuda_status(e, "pkg_reserve_memory");
  return PKG_OK;
}

extern "C" int pkg_trim_memory(size_t keep_bytes) {
  cudaMemPool_t p = lib_pool();
  if (!p) {
    set_last_error("could not create the library memory pool");
    return PKG_ERR_CUDA;
  }
  PK_CUDA(cudaMemPoolTrimTo(p, keep_bytes));
  return PKG_OK;
}

extern "C" const char* pkg_last_error(void) { return g_last_error; }

extern "C" int pkg_release_thread_resources(void) {
  t_res.release();
  return PKG_OK;
}

extern "C" int pkg_thread_resource_bytes(size_t* host_bytes, size_t* device_bytes) {
  PK_REQUIRE(host_bytes && device_bytes, "null output");
  thread_resource_totals(host_bytes, device_bytes);
  return PKG_OK;
}

extern "C" int pkg_version(void) { return 100; }

extern "C" uint64_t pkg_kernel_launches(void) { return g_launches.load(); }

extern "C" int pkg_sample_fr(uint64_t seed, size_t n, uint64_t* out, int mont) {
  if (n && !out) {
    set_last_error("pkg_sample_fr: null output");
    return PKG_ERR_INVALID_ARGUMENT;
  }
  const uint32_t key[8] = {(uint32_t)seed, (uint32_t)(seed >> 32), 0, 0, 0, 0, 0, 0};
  uint64_t counter = 0;
  size_t got = 0;
  uint32_t blk[16];
  while (got < n) {
    chacha20_block(key, counter++, blk);
    for (int h = 0; h < 2 && got < n; h++) {
      HostFr v;
      for (int i = 0; i < 4; i++)
        v.l[i] = (uint64_t)blk[8 * h + 2 * i] | ((uint64_t)blk[8 * h + 2 * i + 1] << 32);
      v.l[3] &= 0x3fffffffffffffffULL;
      if (!v.is_canonical()) continue;
      if (mont) v = HostFr::to_mont(v);
      memcpy(out + 4 * got, v.l, 32);
      got++;
    }
  }
  return PKG_OK;
}

namespace pk {
__device__ __forceinline__ uint32_t rotl32_dev(uint32_t x, int n) {
  return (x << n) | (x >> (32 - n));
}

// ChaCha20 block (RFC 8439 layout: constants, 8 key words, 64-bit counter,
// nonce words) with key = (k0, k1, 0, ...) and nonce word 14 = nonce.
__device__ void chacha20_block_dev(uint32_t k0, uint32_t k1, uint64_t counter, uint32_t nonce,
                                   uint32_t out[16]) {
  const uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                          k0, k1, 0u, 0u, 0u, 0u, 0u, 0u,
                          (uint32_t)counter, (uint32_t)(counter >> 32), nonce, 0u};
  uint32_t x[16];
#pragma unroll
  for (int i = 0; i < 16; i++) x[i] = s[i];
#define PK_QR(a, b, c, d)                                   \
  a += b; d ^= a; d = rotl32_dev(d, 16);                    \
  c += d; b ^= c; b = rotl32_dev(b, 12);                    \
  a += b; d ^= a; d = rotl32_dev(d, 8);                     \
  c += d; b ^= c; b = rotl32_dev(b, 7);
#pragma unroll 1
  for (int r = 0; r < 10; r++) {
    PK_QR(x[0], x[4], x[8], x[12]);
    PK_QR(x[1], x[5], x[9], x[13]);
    PK_QR(x[2], x[6], x[10], x[14]);
    PK_QR(x[3], x[7], x[11], x[15]);
    PK_QR(x[0], x[5], x[10], x[15]);
    PK_QR(x[1], x[6], x[11], x[12]);
    PK_QR(x[2], x[7], x[8], x[13]);
    PK_QR(x[3], x[4], x[9], x[14]);
  }
#undef PK_QR
#pragma unroll
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// out[i] = lo + hi 2^253 mod p (Montgomery) from ChaCha20 block start + i,
// as two products on the FP64 pipe: lo * R^2 and hi * (2^253 R^2), each
// times R^-1 (lo, hi < 2^253 < p).
__global__ void sample_indexed_kernel(uint32_t k0, uint32_t k1, uint64_t start, size_t n, Fr r2,
                                      Fr t253r2, uint64_t* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t b[16];
    chacha20_block_dev(k0, k1, start + i, 1u, b);
    Fr lo, hi;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      lo.v[j] = b[j];
      hi.v[j] = b[8 + j];
    }
    lo.v[7] &= 0x1fffffffu;
    hi.v[7] &= 0x1fffffffu;
    fr_store(out, i, fr_add(fr_mul_f64(lo, r2), fr_mul_f64(hi, t253r2)));
  }
}
}  // namespace pk

extern "C" int pkg_sample_fr_indexed(uint64_t seed, uint64_t start, size_t n, uint64_t* out,
                                     pkg_stream_t stream) {
  if (n == 0) return PKG_OK;
  PK_REQUIRE(out && aligned16(out), "null or unaligned output");
  HostFr one, two253;
  one.l[0] = 1;
  two253.l[3] = uint64_t(1) << 61;
  // x R^2 mod p as raw limbs: to_mont applied twice
  const HostFr r2h = HostFr::to_mont(HostFr::to_mont(one));
  const HostFr th = HostFr::to_mont(HostFr::to_mont(two253));
  Fr r2, t253r2;
  memcpy(r2.v, r2h.l, 32);
  memcpy(t253r2.v, th.l, 32);
  const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  sample_indexed_kernel<<<grid, 256, 0, as_stream(stream)>>>((uint32_t)seed,
                                                              (uint32_t)(seed >> 32), start, n,
                                                              r2, t253r2, out);
  PK_CHECK_LAUNCH("sample_indexed_kernel");
  return PKG_OK;
}

extern "C" int pkg_measure_imad_rate(double* instr_per_second) {
  if (!instr_per_second) return PKG_ERR_INVALID_ARGUMENT;
  uint32_t* sink = nullptr;
  PK_CUDA(cudaMalloc(&sink, 1024 * sizeof(uint32_t)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = sm_count() * 8, iters = 4096;
  imad_rate_kernel<<<blocks, threads>>>(sink, 1u, 64);  // warm-up
  cudaEventRecord(e0);
  imad_rate_kernel<<<blocks, threads>>>(sink, 2u, iters);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return cuda_status(err, "imad_rate_kernel");
  double instr = (double)blocks * threads * iters * 8.0 * 8.0;
  *instr_per_second = instr / (ms * 1e-3);
  return PKG_OK;
}

extern "C" int pkg_measure_dfma_rate(double* instr_per_second) {
  if (!instr_per_second) return PKG_ERR_INVALID_ARGUMENT;
  double* sink = nullptr;
  PK_CUDA(cudaMalloc(&sink, 1024 * sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = sm_count() * 8, iters = 4096;
  dfma_rate_kernel<<<blocks, threads>>>(sink, 0.999999, 1e-7, 64);  // warm-up
  cudaEventRecord(e0);
  dfma_rate_kernel<<<blocks, threads>>>(sink, 0.999999, 1e-7, iters);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return cuda_status(err, "dfma_rate_kernel");
  double instr = (double)blocks * threads * iters * 8.0 * 8.0;
  *instr_per_second = instr / (ms * 1e-3);
  return PKG_OK;
}

extern "C" int pkg_copy_to_host(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return PKG_OK;
  PK_REQUIRE(dst && src, "null pointer");
  PK_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
  return PKG_OK;
}
