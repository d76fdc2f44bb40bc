// host_stage.cuh -- the staging engine behind the pkg_host_* entry points
// (the host-slice seams of the reference: RSFr::interleaved_encode,
// HashEngine::hash_many, ntt_nr / intt_rn on &mut [Fr]).
//
// Those calls receive pageable host memory and must return results in host
// memory.  Per device the stager keeps
//   * a grow-only device workspace (no cudaMalloc / cudaFree per call: a
//     cudaFree synchronises the device and unmaps pages),
//   * a ring of pinned staging chunks, filled / drained by a small pool of
//     host threads so the pageable <-> pinned copies run at several times
//     one core's memcpy bandwidth, and overlapped with the DMA of the
//     neighbouring chunk on the stager's own stream.
// Calls on one device are serialised by the stager's mutex (each pkg_host_*
// call is synchronous anyway); calls on different devices run in parallel.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

namespace pk {

struct HostSegment {
  const void* src;  // host
  size_t bytes;
};

class HostStager {
 public:
  // The stager of the current device (created on first use).
  static HostStager& current();
  std::mutex& mutex() { return mu_; }
  cudaStream_t stream() const { return stream_; }
  // Device workspace of at least `bytes` (grow-only, 256-byte aligned);
  // valid until the next workspace() call on this stager.
  int workspace(size_t bytes, uint8_t** out);
  // Host segments, concatenated, -> device dst.  Returns a pkg status.
  int h2d(uint8_t* dst, const HostSegment* segs, size_t nsegs);
  int h2d(uint8_t* dst, const void* src, size_t bytes) {
    HostSegment s{src, bytes};
    return h2d(dst, &s, 1);
  }
  // Device src -> host dst (after the work queued on stream()).
  int d2h(void* dst, const uint8_t* src, size_t bytes);
  // Set up the stream, pinned chunks and events if not done yet.
  int ensure();
  // Make `consumer` wait for every copy queued so far on stream().
  int handoff(cudaStream_t consumer);

 private:
  HostStager() = default;
  int init();
  std::mutex mu_;
  int device_ = -1;
  cudaStream_t stream_ = nullptr;
  static constexpr int kSlots = 3;
  static constexpr size_t kChunk = size_t(8) << 20;
  uint8_t* pinned_[kSlots] = {};
  cudaEvent_t done_[kSlots] = {};
  cudaEvent_t handoff_ = nullptr;
  uint8_t* ws_ = nullptr;
  size_t ws_bytes_ = 0;
};

// Copy bytes with the stager's host thread pool (used for pageable <->
// pinned copies; falls back to one memcpy for small sizes).
void parallel_memcpy(void* dst, const void* src, size_t bytes);

}  // namespace pk
