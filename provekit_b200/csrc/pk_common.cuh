// pk_common.cuh -- status codes, last-error plumbing and launch helpers shared
// by every translation unit of libprovekit_b200.
//
// Error conventions mirror the reference's FFI layer
// (tooling/provekit-ffi/src/ffi.rs:29-95): every entry point returns an int
// status (0 = ok, negative = error), nothing throws across the C ABI, and a
// thread-local message is readable through pkg_last_error().
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/provekit_b200.h"

namespace pk {

void set_last_error(const char* fmt, ...);
void clear_last_error();

inline int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PKG_OK;
  set_last_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? PKG_ERR_OUT_OF_MEMORY : PKG_ERR_CUDA;
}

#define PK_CUDA(call)                                              \
  do {                                                             \
    cudaError_t _e = (call);                                       \
    if (_e != cudaSuccess) return ::pk::cuda_status(_e, #call);    \
  } while (0)

void count_launch();
// Subtract n launches from the counter (n may wrap to add: 0 - n).
void count_launches_undo(uint64_t n);

#define PK_CHECK_LAUNCH(name) \
  do {                        \
    ::pk::count_launch();     \
    PK_CUDA(cudaGetLastError()); \
  } while (0)

#define PK_REQUIRE(cond, ...)                  \
  do {                                         \
    if (!(cond)) {                             \
      ::pk::set_last_error(__VA_ARGS__);       \
      return PKG_ERR_INVALID_ARGUMENT;         \
    }                                          \
  } while (0)

inline bool is_pow2(size_t n) { return n && !(n & (n - 1)); }
inline int log2_exact(size_t n) {
  int k = 0;
  while ((size_t(1) << k) < n) k++;
  return k;
}
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
inline cudaStream_t as_stream(pkg_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

// Device -> host reads of small results (sumcheck sums, roots, openings)
// through a per-thread pinned bounce buffer, then a stream synchronisation:
// a copy into pageable memory goes through the driver's staging buffer, and
// the proof path makes dozens of these per proof.  Reads that do not fit
// the bounce buffer are copied directly.
struct HostRead {
  void* dst;
  const void* src;
  size_t bytes;
};
int read_small(const HostRead* reads, int n, cudaStream_t s);

// Per host thread: a mapped pinned buffer of kFusedSlotFr Fr that fused
// reductions (reduce.cuh's RedOut with a ticket) write their sums to, and a
// device counter on the current device for their tickets.  One of each per
// thread is enough because every user launches its fused reductions in
// stream order on one stream and synchronises before returning, so a
// thread's fused launches never run at the same time.  Builds with
// -DPK_DEBUG_FUSED check that rule: a fused use that begins while the
// thread's previous one has not synchronised fails.
struct FusedSlots {
  uint64_t* host;    // the buffer, as the host reads it
  uint64_t* dev;     // the same buffer, as kernels write it
  unsigned* ticket;  // zero between launches
  uint64_t* part;    // device partials: 3 Fr for each of up to 4 CTAs per SM
  unsigned long long* pow;  // device word of the PoW search (its own, after the partials)
};
constexpr size_t kFusedSlotFr = 64;
int fused_slots(FusedSlots* f);
// A spare 32-bit word of the thread's mapped pinned slots buffer (after the
// slots and the completion word): a caller may copy a device flag there with
// cudaMemcpyAsync and read it after a later synchronising read on the same
// stream (fused_read, read_small), which implies the copy completed.
int fused_aux_word(uint32_t** word);
// The completion number for the next fused launch of this thread on the
// current device (its RedOut's seq; never 0).
unsigned fused_next_seq();
// Waits until the thread's last fused launch has written its sums (its
// completion word, else the stream's completion), then copies bytes of the
// thread's slots to dst.  Work enqueued after that launch may still run.
int fused_read(void* dst, const FusedSlots& f, size_t bytes, cudaStream_t s);

// Per host thread and device: a grow-only pinned staging buffer and an event
// that marks the last copy into it (the WHIR prover's STIR openings).
// Waits for that event before handing the buffer out again.
struct PinnedStage {
  uint8_t* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t copied = nullptr;
};
int pinned_stage(size_t bytes, PinnedStage** out);

// The per-thread resources above (fused slots, their device counters and
// partials, the read_small bounce buffer, the pinned stages) are owned by one
// thread_local object: released when the thread exits, or earlier by
// pkg_release_thread_resources.  Live totals over all threads, for
// pkg_thread_resource_bytes.
void thread_resource_totals(size_t* host_bytes, size_t* device_bytes);

// Allocates the calling thread's per-thread resources on the current device
// now (fused slots and their device block, the bounce buffer, a pinned stage
// of at least stage_bytes), so that a long-lived thread's first proof does
// not pay for them.
int warm_thread_resources(size_t stage_bytes);

inline int read_small(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  const HostRead r{dst, src, bytes};
  return read_small(&r, 1, s);
}

// Stream-ordered scratch allocation (cudaMallocAsync), freed on scope exit
// in stream order.
// The library's stream-ordered memory pool on the current device (created on
// first use).  Unlike the device's default pool (release threshold 0, which
// hands freed memory back to the driver at every synchronisation and makes
// the next allocation map it again), it keeps what it has grown to until
// pkg_trim_memory.  Returns nullptr if the pool cannot be created.
cudaMemPool_t lib_pool();

// Stream-ordered scratch from lib_pool(), freed (stream-ordered) on scope exit.
struct Scratch {
  void* ptr = nullptr;
  cudaStream_t stream = nullptr;
  Scratch() = default;
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  int alloc(size_t bytes, cudaStream_t s) {
    stream = s;
    if (bytes == 0) return PKG_OK;
    cudaMemPool_t pool = lib_pool();
    if (!pool) {
      set_last_error("could not create the library memory pool");
      return PKG_ERR_CUDA;
    }
    PK_CUDA(cudaMallocFromPoolAsync(&ptr, bytes, pool, s));
    return PKG_OK;
  }
  ~Scratch() {
    if (ptr) cudaFreeAsync(ptr, stream);
  }
};

}  // namespace pk
