// host_stage.cu -- pinned, pipelined staging for the host-slice entry points.
#include "host_stage.cuh"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <thread>
#include <vector>

#include <unistd.h>

#include "pk_common.cuh"

namespace pk {

namespace {

// A fixed pool of host threads that split one memcpy between them.  Leaked on
// purpose: its threads park on a condition variable and end with the process.
class CopyPool {
 public:
  CopyPool() : owner_(getpid()) {
    unsigned hw = std::thread::hardware_concurrency();
    nthreads_ = (int)std::min(8u, hw > 2 ? hw / 2 : 1u);
    for (int i = 0; i < nthreads_; i++) std::thread([this, i] { worker(i); }).detach();
  }
  void run(void* dst, const void* src, size_t bytes) {
    // A forked child has none of the parent's threads: copy on the caller.
    if (bytes < (size_t(1) << 20) || nthreads_ < 2 || getpid() != owner_) {
      std::memcpy(dst, src, bytes);
      return;
    }
    std::lock_guard<std::mutex> one(run_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    dst_ = static_cast<uint8_t*>(dst);
    src_ = static_cast<const uint8_t*>(src);
    bytes_ = bytes;
    pending_ = nthreads_;
    gen_++;
    cv_.notify_all();
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }

 private:
  void worker(int idx) {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return gen_ != seen; });
      seen = gen_;
      uint8_t* dst = dst_;
      const uint8_t* src = src_;
      const size_t bytes = bytes_;
      lk.unlock();
      size_t part = (bytes / nthreads_ + 4095) & ~size_t(4095);
      size_t off = part * idx;
      if (off < bytes) std::memcpy(dst + off, src + off, std::min(part, bytes - off));
      lk.lock();
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }
  const pid_t owner_;
  int nthreads_ = 0;
  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  uint64_t gen_ = 0;
  int pending_ = 0;
  uint8_t* dst_ = nullptr;
  const uint8_t* src_ = nullptr;
  size_t bytes_ = 0;
};

CopyPool& pool() {
  static CopyPool* p = new CopyPool();
  return *p;
}

std::mutex g_stagers_mu;
HostStager* g_stagers[64] = {};

}  // namespace

void parallel_memcpy(void* dst, const void* src, size_t bytes) { pool().run(dst, src, bytes); }

int HostStager::init() {
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  if (!stream_) PK_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (int i = 0; i < kSlots; i++) {
    if (!pinned_[i])
      PK_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&pinned_[i]), kChunk, cudaHostAllocDefault));
    if (!done_[i]) PK_CUDA(cudaEventCreateWithFlags(&done_[i], cudaEventDisableTiming));
  }
  if (!handoff_) PK_CUDA(cudaEventCreateWithFlags(&handoff_, cudaEventDisableTiming));
  device_ = dev;  // set last: a failed set-up is retried by the next call
  return PKG_OK;
}

int HostStager::ensure() { return device_ < 0 ? init() : PKG_OK; }

int HostStager::handoff(cudaStream_t consumer) {
  PK_CUDA(cudaEventRecord(handoff_, stream_));
  PK_CUDA(cudaStreamWaitEvent(consumer, handoff_, 0));
  return PKG_OK;
}

HostStager& HostStager::current() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_stagers_mu);
  HostStager*& s = g_stagers[dev & 63];
  if (!s) s = new HostStager();
  return *s;
}

int HostStager::workspace(size_t bytes, uint8_t** out) {
  int rc = ensure();
  if (rc) return rc;
  if (bytes > ws_bytes_) {
    if (ws_) {
      PK_CUDA(cudaStreamSynchronize(stream_));
      cudaFree(ws_);
      ws_ = nullptr;
      ws_bytes_ = 0;
    }
    const size_t want = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    PK_CUDA(cudaMalloc(&ws_, want));
    ws_bytes_ = want;
  }
  *out = ws_;
  return PKG_OK;
}

int HostStager::h2d(uint8_t* dst, const HostSegment* segs, size_t nsegs) {
  size_t seg = 0, seg_off = 0, off = 0;
  int slot = 0;
  while (seg < nsegs) {
    if (segs[seg].bytes == seg_off) {
      seg++;
      seg_off = 0;
      continue;
    }
    PK_CUDA(cudaEventSynchronize(done_[slot]));  // the slot's previous DMA has read it
    size_t fill = 0;
    while (fill < kChunk && seg < nsegs) {
      const size_t take = std::min(kChunk - fill, segs[seg].bytes - seg_off);
      parallel_memcpy(pinned_[slot] + fill, static_cast<const uint8_t*>(segs[seg].src) + seg_off,
                      take);
      fill += take;
      seg_off += take;
      if (seg_off == segs[seg].bytes) {
        seg++;
        seg_off = 0;
      }
    }
    PK_CUDA(cudaMemcpyAsync(dst + off, pinned_[slot], fill, cudaMemcpyHostToDevice, stream_));
    PK_CUDA(cudaEventRecord(done_[slot], stream_));
    off += fill;
    slot = (slot + 1) % kSlots;
  }
  return PKG_OK;
}

int HostStager::d2h(void* dst, const uint8_t* src, size_t bytes) {
  const size_t n = (bytes + kChunk - 1) / kChunk;
  auto len = [&](size_t c) { return std::min(kChunk, bytes - c * kChunk); };
  auto issue = [&](size_t c) -> int {
    const int slot = (int)(c % kSlots);
    PK_CUDA(cudaMemcpyAsync(pinned_[slot], src + c * kChunk, len(c), cudaMemcpyDeviceToHost,
                            stream_));
    PK_CUDA(cudaEventRecord(done_[slot], stream_));
    return PKG_OK;
  };
  for (size_t c = 0; c < std::min(n, (size_t)kSlots); c++) {
    int rc = issue(c);
    if (rc) return rc;
  }
  for (size_t c = 0; c < n; c++) {
    const int slot = (int)(c % kSlots);
    PK_CUDA(cudaEventSynchronize(done_[slot]));
    parallel_memcpy(static_cast<uint8_t*>(dst) + c * kChunk, pinned_[slot], len(c));
    if (c + kSlots < n) {
      int rc = issue(c + kSlots);
      if (rc) return rc;
    }
  }
  return PKG_OK;
}

}  // namespace pk
