// reduce.cuh -- block-wide sums of field elements and the grid-size helpers
// shared by the reduction kernels (sumcheck, dot products, WHIR rounds).
//
// Each thread accumulates a grid-stride slice; warps combine with
// __shfl_down_sync (8 limbs per element, field additions), warps combine
// through shared memory, and one partial per CTA goes to a small scratch
// array that a single-CTA kernel sums.  Field addition is exact, so the
// result does not depend on the reduction order.
#pragma once
#include <algorithm>

#include "fr.cuh"
#include "fr_f64.cuh"
#include "pk_common.cuh"

namespace pk {

constexpr int kRedThreads = 256;

__device__ __forceinline__ Fr shfl_down(const Fr& x, int off) {
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = __shfl_down_sync(0xffffffffu, x.v[i], off);
  return r;
}

// Block-wide sum of K field elements per thread; thread 0 gets the result.
template <int K>
__device__ __forceinline__ void block_sum(Fr (&v)[K]) {
  __shared__ Fr warp_sums[kRedThreads / 32][K];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = fr_add(v[k], shfl_down(v[k], off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; k++) warp_sums[warp][k] = v[k];
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = lane < nw ? warp_sums[lane][k] : fr_zero();
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = fr_add(v[k], shfl_down(v[k], off));
  }
}

// Where a reduction kernel's CTAs leave their sums.  part: one partial per
// CTA (K Fr each), summed by sum_partials_kernel.  With a ticket, the kernel
// finishes the sum itself: every CTA takes a ticket after storing its
// partial, and the CTA that takes the last one adds all partials, writes the
// K sums to out (device or mapped host memory) and resets the counter for the
// next launch -- one launch instead of two, no copy when out is mapped.
//
// A fused launch also announces its completion to the host: after writing
// the sums, the last CTA stores seq (fused_next_seq(), nonzero) into a word
// of mapped host memory whose device address sits in the ticket's block
// (ticket + 2, see fused_slots), so fused_read can poll that word instead of
// waiting for the stream.
struct RedOut {
  uint64_t* part;
  unsigned* ticket;  // nullptr: partials only
  uint64_t* out;
  unsigned seq;      // 0: no completion word
};

// 32 bytes through L2 only: partials other CTAs wrote during this launch.
__device__ __forceinline__ Fr fr_load_cg(const uint64_t* base, size_t idx) {
  const uint4* q = reinterpret_cast<const uint4*>(base + 4 * idx);
  const uint4 a = __ldcg(q), b = __ldcg(q + 1);
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}

// The end of a reduction kernel: block sum, the CTA's partial, and with a
// ticket the last CTA's final sum.  Every thread of the CTA calls it.
// scale (or nullptr): each CTA sum is multiplied by it (Montgomery product)
// before it is stored -- the 2^8 that lazily reduced sums (fr_lazy.cuh) owe.
template <int K>
__device__ __forceinline__ void block_finish(Fr (&v)[K], const RedOut& ro,
                                             const Fr* scale = nullptr) {
  __shared__ bool last;
  block_sum<K>(v);
  if (threadIdx.x == 0) {
    if (scale)
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = fr_mul_f64(v[k], *scale);
#pragma unroll
    for (int k = 0; k < K; k++) fr_store(ro.part, (size_t)blockIdx.x * K + k, v[k]);
    if (ro.ticket) {
      __threadfence();
      last = atomicAdd(ro.ticket, 1u) == gridDim.x - 1;
    }
  }
  if (!ro.ticket) return;
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = fr_zero();
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = fr_add(v[k], fr_load_cg(ro.part, (size_t)i * K + k));
  block_sum<K>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) fr_store(ro.out, k, v[k]);
    *ro.ticket = 0u;
    if (ro.seq) {
      volatile unsigned* word = *reinterpret_cast<unsigned* const*>(ro.ticket + 2);
      __threadfence_system();  // the sums before the completion word
      *word = ro.seq;
    }
  }
}

template <int K>
__global__ void __launch_bounds__(kRedThreads) sum_partials_kernel(const uint64_t* __restrict__ part,
                                                                 int nparts,
                                                                 uint64_t* __restrict__ out) {
  Fr v[K];
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = fr_zero();
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = fr_add(v[k], fr_load(part, (size_t)i * K + k));
  block_sum<K>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) fr_store(out, k, v[k]);
}

// CTAs for a reduction over n items (at most 4 per SM).
inline int red_grid(size_t n) {
  size_t b = (n + kRedThreads - 1) / kRedThreads;
  return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sm_count() * 4));
}
// CTAs of 256 threads for an element-wise kernel over n items (grid-stride).
inline int ew_grid(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sm_count() * 32));
}

}  // namespace pk
