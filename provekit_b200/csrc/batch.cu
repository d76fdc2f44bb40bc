// batch.cu -- the batched form: many independent jobs of uneven sizes, each
// an NTT, a WHIR commit of its coefficients (RS encode at rate 1/4 over 8
// interleaved messages + Skyscraper tree) and a Spartan zk-sumcheck, run as
// one CUDA graph of grouped kernels.
//
// Every phase is ONE launch over all jobs: a small device table maps each CTA
// (or each element) to its job, so 256 jobs cost the same number of launches
// as one.  NTT passes take their radix (K stages) and CTA shape at run time
// per job; the autotuner (pkg_batch_tune) sweeps the largest radix 2^4..2^11,
// the elements per CTA and the butterflies each thread runs per stage (1, 2
// or 4: the CTA size for a given tile).  The sumcheck's Fiat-Shamir transcript and the
// round-polynomial bookkeeping run on the device (one thread per job), so a
// whole batch has no host round trip and is captured once and replayed.
//
// Results are bit-identical to running each job alone through pkg_ntt_nr,
// pkg_whir_commit and pkg_spartan_sumcheck.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "fr.cuh"
#include "fr_host.hpp"
#include "ntt_internal.cuh"
#include "pk_common.cuh"
#include "skyscraper.cuh"
#include "sumcheck_device.cuh"

namespace pk {

constexpr int kMsgs = 8;         // RS messages per job (folding factor 3)
constexpr int kLogInvRate = 2;   // rate 1/4
constexpr int kMaxM0 = 30;
constexpr int kScThreads = 256;  // sumcheck round CTA size
constexpr int kScCtaCap = 64;    // CTAs per job per round

struct PassDesc {  // one job's share of one grouped NTT pass
  uint64_t* data;
  uint64_t U;
  uint64_t cta_begin;
  uint32_t log_u, K, T, log_t, mode_b, pad;
  // Where a job's first pass reads its input: 0 = data itself, 1 = src (the
  // coefficients, same indices), 2 = src through the RS-encode layout of
  // kMsgs messages of src_n / kMsgs (the transpose and 4-coset replication).
  const uint64_t* src;
  uint64_t src_n;
  uint32_t src_kind, pad2;
};

struct RangeDesc {  // job j owns [begin, begin + count) of a grouped launch
  uint64_t begin, count;
  const uint64_t* in;  // phase-specific input
  uint8_t* out;        // phase-specific output
  uint32_t job, pad;
};

struct ScState {  // device-side sumcheck state of one job
  Fr tl, tr;      // transcript (canonical)
  Fr rho, saved, sum_g, blinding_eval;
  Fr r[kMaxM0], alpha[kMaxM0];
  Fr coeffs[kMaxM0][4];
  Fr g[kMaxM0][4];
  Fr wb[kMaxM0][4];
  Fr domain;  // canonical
  uint32_t m0, pad[7];
};

struct JobDev {
  uint64_t *coeffs, *ntt, *cw, *a, *b, *c, *eq, *eq_hi, *eq_lo, *part;
  uint8_t* layers;
  uint64_t n, cw_rows, part_begin;
  uint32_t log_n, m0, nhi, nlo;
};

__device__ __forceinline__ uint32_t find_desc(const uint64_t* begins, uint32_t n, uint64_t key) {
  uint32_t lo = 0, hi = n;  // last i with begins[i] <= key
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (begins[mid] <= key) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Shared memory as two planes of 16-byte halves (see ntt_pass_kernel).
__device__ __forceinline__ Fr sm_get(const uint4* sm, int E, int i) {
  uint4 a = sm[i], b = sm[E + i];
  Fr x;
  x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
  x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
  return x;
}
__device__ __forceinline__ void sm_put(uint4* sm, int E, int i, const Fr& x) {
  sm[i] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  sm[E + i] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// ---- grouped NTT pass: the ntt_pass_kernel index scheme with run-time K ----
__global__ void __launch_bounds__(512) batch_ntt_pass_kernel(const PassDesc* __restrict__ descs,
                                                            const uint64_t* __restrict__ begins,
                                                            uint32_t ndesc,
                                                            const uint64_t* __restrict__ roots) {
  extern __shared__ uint4 sm[];
  const PassDesc d = descs[find_desc(begins, ndesc, blockIdx.x)];
  const int K = (int)d.K, R = 1 << K, T = (int)d.T, log_t = (int)d.log_t, log_u = (int)d.log_u;
  const int E = R * T;
  const uint64_t U = d.U;
  const uint64_t l0 = (uint64_t)(blockIdx.x - d.cta_begin) * T;
  uint64_t high_a = 0, u0 = 0;
  if (!d.mode_b) {
    high_a = l0 / U;
    u0 = l0 - high_a * U;
  }
  uint64_t* data = d.data;
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    uint64_t g;
    int sidx;
    if (!d.mode_b) {
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
    const uint4* in;
    if (d.src_kind == 0) {
      in = reinterpret_cast<const uint4*>(data + 4 * g);
    } else if (d.src_kind == 1) {
      in = reinterpret_cast<const uint4*>(d.src + 4 * g);
    } else {  // row x of each n-element coset block holds messages[x % 8][x / 8]
      const uint64_t x = g & (d.src_n - 1);
      in = reinterpret_cast<const uint4*>(d.src + 4 * ((x % kMsgs) * (d.src_n / kMsgs) + x / kMsgs));
    }
    sm[sidx] = in[0];      // low 16 bytes: plane 0
    sm[E + sidx] = in[1];  // high 16 bytes: plane 1
  }
  __syncthreads();
  for (int s = 0; s < K; s++) {
    const int log_h = K - 1 - s;
    for (int b = threadIdx.x; b < (E >> 1); b += blockDim.x) {
      int ll = b & (T - 1);
      int p = b >> log_t;
      int grp = p >> log_h;
      int pos = p & ((1 << log_h) - 1);
      int j0 = (grp << (log_h + 1)) + pos;
      int j1 = j0 + (1 << log_h);
      uint64_t high = d.mode_b ? ((l0 + ll) >> log_u) : high_a;
      Fr tw = fr_load_ro(roots, (high << s) | (uint64_t)grp);
      int i0 = j0 * T + ll, i1 = j1 * T + ll;
      Fr x0 = sm_get(sm, E, i0), x1 = sm_get(sm, E, i1);
      Fr m = fr_mul_f64(tw, x1);
      sm_put(sm, E, i0, fr_add(x0, m));
      sm_put(sm, E, i1, fr_sub(x0, m));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    uint64_t g;
    int sidx;
    if (!d.mode_b) {
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

// ---- grouped element-wise phases ------------------------------------------
// Fr copy: out[i] = in[i] for each range.
__global__ void batch_copy_kernel(const RangeDesc* __restrict__ rd, const uint64_t* __restrict__ begins,
                                  uint32_t nd, uint64_t total) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const RangeDesc d = rd[find_desc(begins, nd, o)];
    const uint64_t i = o - d.begin;
    fr_store(reinterpret_cast<uint64_t*>(d.out), i, fr_load_ro(d.in, i));
  }
}

// Merkle leaves: leaf i = codeword row i (8 Fr), canonical encoding.
__global__ void batch_leaves_kernel(const RangeDesc* __restrict__ rd,
                                    const uint64_t* __restrict__ begins, uint32_t nd,
                                    uint64_t total) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const RangeDesc d = rd[find_desc(begins, nd, o)];
    const uint64_t i = o - d.begin;
    Fr acc = fr_from_mont(fr_load_ro(d.in, i * kMsgs));
#pragma unroll 1
    for (int k = 1; k < kMsgs; k++) acc = sky_compress(acc, fr_from_mont(fr_load_ro(d.in, i * kMsgs + k)));
    fr_store(reinterpret_cast<uint64_t*>(d.out), i, acc);
  }
}

// One tree level for every job that still has one: out[i] = compress(in[2i], in[2i+1]).
__global__ void batch_level_kernel(const RangeDesc* __restrict__ rd,
                                   const uint64_t* __restrict__ begins, uint32_t nd, uint64_t total) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const RangeDesc d = rd[find_desc(begins, nd, o)];
    const uint64_t i = o - d.begin;
    Fr l = fr_load_ro(d.in, 2 * i), r = fr_load_ro(d.in, 2 * i + 1);
    fr_store(reinterpret_cast<uint64_t*>(d.out), i, sky_compress(l, r));
  }
}

// ---- device sumcheck ------------------------------------------------------
// Start: transcript init, r challenges, eq half tables, sum_g, rho.
__global__ void batch_sc_start_kernel(ScState* __restrict__ st, const JobDev* __restrict__ jobs,
                                      uint32_t njobs) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  ScState& s = st[j];
  DevTranscript t;
  t.init(s.domain);
  for (uint32_t i = 0; i < s.m0; i++) s.r[i] = t.squeeze();  // whir_r1cs.rs:529
  Fr g0[4];
  dev_blinding_coeffs(&s.g[0][0], (int)s.m0, 0, s.alpha, g0);
  s.sum_g = fr_add(dev_cubic(g0, fr_zero()), dev_cubic(g0, fr_one_mont()));
  t.absorb(s.sum_g);   // :541
  s.rho = t.squeeze();  // :543
  s.saved = fr_mul_f64(s.rho, s.sum_g);
  s.tl = t.l;
  s.tr = t.r;
}

// eq half tables: hi over r[0..nhi), lo over r[nhi..m0) (same split as
// eq_hypercube_device); grouped over all entries.
__global__ void batch_eq_half_kernel(const RangeDesc* __restrict__ rd,
                                     const uint64_t* __restrict__ begins, uint32_t nd,
                                     uint64_t total, const ScState* __restrict__ st,
                                     const JobDev* __restrict__ jobs) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const RangeDesc d = rd[find_desc(begins, nd, o)];
    const JobDev& jb = jobs[d.job];
    uint64_t x = o - d.begin;
    const bool is_hi = x < (uint64_t(1) << jb.nhi);
    const int nr = is_hi ? (int)jb.nhi : (int)jb.nlo;
    const int r0 = is_hi ? 0 : (int)jb.nhi;
    if (!is_hi) x -= uint64_t(1) << jb.nhi;
    Fr acc = fr_one_mont();
    for (int i = 0; i < nr; i++) {
      const Fr ri = st[d.job].r[r0 + i];
      acc = fr_mul_f64(acc, ((x >> (nr - 1 - i)) & 1) ? ri : fr_sub(fr_one_mont(), ri));
    }
    fr_store(is_hi ? jb.eq_hi : jb.eq_lo, x, acc);
  }
}

__global__ void batch_eq_combine_kernel(const RangeDesc* __restrict__ rd,
                                        const uint64_t* __restrict__ begins, uint32_t nd,
                                        uint64_t total, const JobDev* __restrict__ jobs) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const RangeDesc d = rd[find_desc(begins, nd, o)];
    const JobDev& jb = jobs[d.job];
    const uint64_t x = o - d.begin;
    fr_store(jb.eq, x, fr_mul_f64(fr_load_ro(jb.eq_hi, x >> jb.nlo),
                              fr_load_ro(jb.eq_lo, x & ((uint64_t(1) << jb.nlo) - 1))));
  }
}

__device__ __forceinline__ Fr shfl_down_fr(const Fr& x, int off) {
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.v[i] = __shfl_down_sync(0xffffffffu, x.v[i], off);
  return r;
}

// One sumcheck round for every job with rounds left.  Each CTA belongs to one
// job (descriptor `count` = pairs q, `begin` = first CTA); per-CTA partial
// sums of (f0, f(-1), f(inf)) go to the job's partial slots.
template <bool kFold>
__global__ void __launch_bounds__(kScThreads) batch_sc_round_kernel(
    const RangeDesc* __restrict__ rd, const uint64_t* __restrict__ begins, uint32_t nd,
    const JobDev* __restrict__ jobs, const ScState* __restrict__ st, uint32_t round) {
  const RangeDesc d = rd[find_desc(begins, nd, blockIdx.x)];
  const JobDev& jb = jobs[d.job];
  const uint64_t size = round == 0 ? jb.n : (jb.n >> (round - 1));  // live table length
  const uint64_t q = kFold ? size / 4 : size / 2;
  const uint32_t cta = blockIdx.x - (uint32_t)d.begin;
  const uint32_t nctas = (uint32_t)d.count;
  Fr fold = fr_zero();
  if (kFold) fold = st[d.job].alpha[round - 1];
  uint64_t* const tabs[4] = {jb.a, jb.b, jb.c, jb.eq};
  Fr acc[3] = {fr_zero(), fr_zero(), fr_zero()};
  for (uint64_t j = (uint64_t)cta * blockDim.x + threadIdx.x; j < q;
       j += (uint64_t)nctas * blockDim.x)
    spartan_pair<kFold>(tabs, j, q, fold, acc);
  __shared__ Fr wsum[kScThreads / 32][3];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < 3; k++) acc[k] = fr_add(acc[k], shfl_down_fr(acc[k], off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 3; k++) wsum[warp][k] = acc[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    Fr s3[3] = {fr_zero(), fr_zero(), fr_zero()};
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
#pragma unroll
      for (int k = 0; k < 3; k++) s3[k] = fr_add(s3[k], wsum[w][k]);
#pragma unroll
    for (int k = 0; k < 3; k++) fr_store(jb.part, (uint64_t)cta * 3 + k, s3[k]);
  }
}

// Round bookkeeping for every job still running: sum the CTA partials, build
// the round polynomial with the blinding terms (whir_r1cs.rs:567-609), absorb
// it and squeeze alpha.
__global__ void batch_sc_finish_round_kernel(ScState* __restrict__ st,
                                             const JobDev* __restrict__ jobs, uint32_t njobs,
                                             uint32_t round, const uint32_t* __restrict__ nctas) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  ScState& s = st[j];
  if (round >= s.m0) return;
  const JobDev& jb = jobs[j];
  Fr h[3] = {fr_zero(), fr_zero(), fr_zero()};
  for (uint32_t c = 0; c < nctas[j]; c++)
#pragma unroll
    for (int k = 0; k < 3; k++) h[k] = fr_add(h[k], fr_load(jb.part, (uint64_t)c * 3 + k));
  Fr gp[4];
  dev_blinding_coeffs(&s.g[0][0], (int)s.m0, (int)round, s.alpha, gp);
  Fr cf[4];
  cf[0] = fr_add(h[0], fr_mul_f64(s.rho, gp[0]));
  Fr gem1 = fr_sub(fr_add(fr_sub(gp[0], gp[1]), gp[2]), gp[3]);
  Fr cem1 = fr_add(h[1], fr_mul_f64(s.rho, gem1));
  cf[2] = fr_mul_f64(fr_half_mont(), fr_sub(fr_sub(fr_sub(fr_add(s.saved, cem1), cf[0]), cf[0]), cf[0]));
  cf[3] = fr_add(h[2], fr_mul_f64(s.rho, gp[3]));
  cf[1] = fr_sub(fr_sub(fr_sub(fr_sub(s.saved, cf[0]), cf[0]), cf[3]), cf[2]);
  DevTranscript t;
  t.l = s.tl;
  t.r = s.tr;
#pragma unroll 1
  for (int k = 0; k < 4; k++) {
    s.coeffs[round][k] = cf[k];
    t.absorb(cf[k]);
  }
  s.alpha[round] = t.squeeze();
  s.saved = dev_cubic(cf, s.alpha[round]);
  s.tl = t.l;
  s.tr = t.r;
}

// blinding_eval = <expand_powers::<4>(alpha), w1[offset..]> (whir_r1cs.rs:613-618), absorbed.
__global__ void batch_sc_end_kernel(ScState* __restrict__ st, uint32_t njobs) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  ScState& s = st[j];
  Fr acc = fr_zero();
  for (uint32_t i = 0; i < s.m0; i++) {
    Fr pw = fr_one_mont();
    for (int k = 0; k < 4; k++) {
      acc = fr_add(acc, fr_mul_f64(pw, s.wb[i][k]));
      pw = fr_mul_f64(pw, s.alpha[i]);
    }
  }
  s.blinding_eval = acc;
  DevTranscript t;
  t.l = s.tl;
  t.r = s.tr;
  t.absorb(acc);
  s.tl = t.l;
  s.tr = t.r;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Grouped {  // one grouped launch: descriptor arrays on the device
  uint64_t total = 0;  // elements (or CTAs for CTA-mapped kernels)
  uint32_t n = 0;
  RangeDesc* d_desc = nullptr;
  uint64_t* d_begin = nullptr;
};

struct PassLaunch {
  uint32_t n = 0;
  uint64_t ctas = 0;
  int threads = 32;
  size_t smem = 0;
  PassDesc* d_desc = nullptr;
  uint64_t* d_begin = nullptr;
};

}  // namespace pk

struct pkg_batch {
  std::vector<uint32_t> log_n;
  std::vector<pk::JobDev> jobs;  // host copy of the device job table
  std::vector<pk::ScState> init_state;
  uint8_t* arena = nullptr;      // all job buffers
  pk::JobDev* d_jobs = nullptr;
  pk::ScState* d_state = nullptr;
  pk::ScState* d_state_init = nullptr;
  uint64_t graph_kernels = 0;
  uint32_t* d_nctas = nullptr;
  uint8_t* tables = nullptr;     // descriptor tables (rebuilt by plan())
  size_t tables_bytes = 0;
  const uint64_t* roots = nullptr;
  // the autotuner's choice on a mix of 256 jobs of 2^10..2^22 points as the default plan:
  // radix 2^10, 1024 elements per CTA, 4 butterflies per thread per stage
  // (492.6 ms per batch, against 503 ms with radix 2^8, 256 elements and one
  // butterfly per thread)
  int kmax = 10, log_elems = 10;
  int log_bpt = 2;  // log2 butterflies per thread per stage (CTA size E / 2^(1 + log_bpt))
  // plan
  std::vector<pk::PassLaunch> passes;
  pk::Grouped leaves, eq_half, eq_comb, copy_sc;
  std::vector<pk::Grouped> levels, rounds;
  std::vector<uint64_t> round_ctas;
  uint32_t max_m0 = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace pk {

static inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static void plan_passes(size_t N, size_t M, int t_begin, int t_end, int kmax, int log_elems,
                        uint64_t* data, const uint64_t* src, uint64_t src_n, uint32_t src_kind,
                        std::vector<std::vector<PassDesc>>& out) {
  int total = t_end - t_begin;
  if (total <= 0) return;
  int np = (total + kmax - 1) / kmax;
  int t = t_begin;
  for (int pi = 0; pi < np; pi++) {
    int K = (total - (t - t_begin) + (np - pi) - 1) / (np - pi);
    int B = log2_exact(N) - t - K;
    uint64_t U = (uint64_t(1) << B) * M;
    uint64_t lines = (uint64_t(1) << t) * U;
    int log_tgt = log_elems > K ? log_elems - K : 0;
    uint64_t T = uint64_t(1) << log_tgt;
    if (T > lines) T = lines & (~lines + 1);
    uint32_t mode_b = 0, log_u = 0;
    if (is_pow2(U) && U < T) {
      mode_b = 1;
      log_u = log2_exact(U);
    } else {
      uint64_t pu = U & (~U + 1);
      if (T > pu) T = pu;
    }
    PassDesc d;
    d.data = data;
    d.U = U;
    d.cta_begin = lines / T;  // CTA count; turned into a begin offset later
    d.log_u = log_u;
    d.K = (uint32_t)K;
    d.T = (uint32_t)T;
    d.log_t = (uint32_t)log2_exact(T);
    d.mode_b = mode_b;
    d.pad = 0;
    d.src = pi == 0 ? src : nullptr;
    d.src_n = src_n;
    d.src_kind = pi == 0 ? src_kind : 0;
    d.pad2 = 0;
    if ((int)out.size() <= pi) out.resize(pi + 1);
    out[pi].push_back(d);
    t += K;
  }
}

static int upload_grouped(pkg_batch* b, std::vector<RangeDesc>& v, Grouped& g, uint8_t*& cursor) {
  g.n = (uint32_t)v.size();
  g.total = 0;
  std::vector<uint64_t> begins(v.size());
  for (size_t i = 0; i < v.size(); i++) {
    v[i].begin = g.total;
    begins[i] = g.total;
    g.total += v[i].count;
  }
  g.d_desc = reinterpret_cast<RangeDesc*>(cursor);
  cursor += align256(sizeof(RangeDesc) * std::max<size_t>(v.size(), 1));
  g.d_begin = reinterpret_cast<uint64_t*>(cursor);
  cursor += align256(8 * std::max<size_t>(v.size(), 1));
  if (!v.empty()) {
    PK_CUDA(cudaMemcpy(g.d_desc, v.data(), sizeof(RangeDesc) * v.size(), cudaMemcpyHostToDevice));
    PK_CUDA(cudaMemcpy(g.d_begin, begins.data(), 8 * v.size(), cudaMemcpyHostToDevice));
  }
  (void)b;
  return PKG_OK;
}

// Build every grouped launch's descriptor tables for the current tuning.
static int batch_plan(pkg_batch* b) {
  const size_t nj = b->jobs.size();
  // NTT passes: the plain NTT of each job and the RS NTT of each codeword.
  std::vector<std::vector<PassDesc>> pass_descs;
  for (size_t j = 0; j < nj; j++) {
    const JobDev& jb = b->jobs[j];
    // first passes read the coefficients directly: the plain NTT's copy and
    // the RS transpose + coset replication are their loads
    plan_passes(jb.n, 1, 0, (int)jb.log_n, b->kmax, b->log_elems, jb.ntt, jb.coeffs, jb.n, 1,
                pass_descs);
    plan_passes(jb.cw_rows, kMsgs, kLogInvRate, log2_exact(jb.cw_rows), b->kmax, b->log_elems,
                jb.cw, jb.coeffs, jb.n, 2, pass_descs);
  }
  std::vector<std::vector<RangeDesc>> lv, rd_rounds;
  std::vector<RangeDesc> lf, eh, ec, csc;
  uint32_t max_m0 = 0;
  for (size_t j = 0; j < nj; j++) {
    const JobDev& jb = b->jobs[j];
    const uint32_t jj = (uint32_t)j;
    lf.push_back({0, jb.cw_rows, jb.cw, jb.layers, jj, 0});
    size_t nodes = jb.cw_rows, off = 0;
    for (int l = 0; nodes > 1; l++) {
      if ((int)lv.size() <= l) lv.resize(l + 1);
      lv[l].push_back({0, nodes / 2, reinterpret_cast<const uint64_t*>(jb.layers + 32 * off),
                       jb.layers + 32 * (off + nodes), jj, 0});
      off += nodes;
      nodes /= 2;
    }
    eh.push_back({0, (uint64_t(1) << jb.nhi) + (uint64_t(1) << jb.nlo), nullptr, nullptr, jj, 0});
    ec.push_back({0, jb.n, nullptr, nullptr, jj, 0});
    // sumcheck tables: a = coeffs, b = NTT output, c = first n codeword entries
    csc.push_back({0, jb.n, jb.coeffs, reinterpret_cast<uint8_t*>(jb.a), jj, 0});
    csc.push_back({0, jb.n, jb.ntt, reinterpret_cast<uint8_t*>(jb.b), jj, 0});
    csc.push_back({0, jb.n, jb.cw, reinterpret_cast<uint8_t*>(jb.c), jj, 0});
    max_m0 = std::max(max_m0, jb.m0);
  }
  b->max_m0 = max_m0;
  b->round_ctas.assign((size_t)max_m0 * nj, 0);
  for (uint32_t r = 0; r < max_m0; r++) {
    rd_rounds.emplace_back();
    for (size_t j = 0; j < nj; j++) {
      const JobDev& jb = b->jobs[j];
      if (r >= jb.m0) continue;
      const uint64_t size = r == 0 ? jb.n : (jb.n >> (r - 1));
      const uint64_t q = r == 0 ? size / 2 : size / 4;
      uint64_t ctas = std::min<uint64_t>((q + kScThreads - 1) / kScThreads, kScCtaCap);
      b->round_ctas[(size_t)r * nj + j] = ctas;
      RangeDesc d = {0, ctas, nullptr, nullptr, (uint32_t)j, 0};
      rd_rounds.back().push_back(d);
    }
  }
  // device descriptor memory
  size_t bytes = 0;
  auto grp = [](size_t n) { return align256(sizeof(RangeDesc) * std::max<size_t>(n, 1)) + align256(8 * std::max<size_t>(n, 1)); };
  for (auto& p : pass_descs) bytes += align256(sizeof(PassDesc) * p.size()) + align256(8 * p.size());
  bytes += grp(lf.size()) + grp(eh.size()) + grp(ec.size()) + grp(csc.size());
  for (auto& l : lv) bytes += grp(l.size());
  for (auto& r : rd_rounds) bytes += grp(r.size());
  if (b->tables) cudaFree(b->tables);
  b->tables = nullptr;
  PK_CUDA(cudaMalloc(&b->tables, bytes));
  b->tables_bytes = bytes;
  uint8_t* cur = b->tables;
  b->passes.clear();
  for (auto& p : pass_descs) {
    PassLaunch pl;
    pl.n = (uint32_t)p.size();
    std::vector<uint64_t> begins(p.size());
    uint64_t acc = 0;
    uint64_t maxe = 0;
    for (size_t i = 0; i < p.size(); i++) {
      uint64_t cnt = p[i].cta_begin;
      p[i].cta_begin = acc;
      begins[i] = acc;
      acc += cnt;
      maxe = std::max<uint64_t>(maxe, (uint64_t(1) << p[i].K) * p[i].T);
    }
    pl.ctas = acc;
    pl.threads =
        (int)std::max<uint64_t>(32, std::min<uint64_t>((maxe / 2) >> b->log_bpt, 512));
    pl.smem = 32 * maxe;
    pl.d_desc = reinterpret_cast<PassDesc*>(cur);
    cur += align256(sizeof(PassDesc) * p.size());
    pl.d_begin = reinterpret_cast<uint64_t*>(cur);
    cur += align256(8 * p.size());
    PK_CUDA(cudaMemcpy(pl.d_desc, p.data(), sizeof(PassDesc) * p.size(), cudaMemcpyHostToDevice));
    PK_CUDA(cudaMemcpy(pl.d_begin, begins.data(), 8 * p.size(), cudaMemcpyHostToDevice));
    b->passes.push_back(pl);
  }
  int rc;
  if ((rc = upload_grouped(b, lf, b->leaves, cur))) return rc;
  if ((rc = upload_grouped(b, eh, b->eq_half, cur))) return rc;
  if ((rc = upload_grouped(b, ec, b->eq_comb, cur))) return rc;
  if ((rc = upload_grouped(b, csc, b->copy_sc, cur))) return rc;
  b->levels.assign(lv.size(), Grouped());
  for (size_t l = 0; l < lv.size(); l++)
    if ((rc = upload_grouped(b, lv[l], b->levels[l], cur))) return rc;
  b->rounds.assign(rd_rounds.size(), Grouped());
  for (size_t r = 0; r < rd_rounds.size(); r++)
    if ((rc = upload_grouped(b, rd_rounds[r], b->rounds[r], cur))) return rc;
  return PKG_OK;
}

static int ew_blocks(uint64_t total) {
  uint64_t g = (total + 255) / 256;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sm_count() * 32));
}

// Enqueue the whole batch on s.
static int batch_enqueue(pkg_batch* b, cudaStream_t s) {
  const uint32_t nj = (uint32_t)b->jobs.size();
  PK_CUDA(cudaMemcpyAsync(b->d_state, b->d_state_init, sizeof(ScState) * nj,
                          cudaMemcpyDeviceToDevice, s));
  for (auto& p : b->passes) {
    if (p.smem > 48 * 1024)
      PK_CUDA(cudaFuncSetAttribute(batch_ntt_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)p.smem));
    batch_ntt_pass_kernel<<<(unsigned)p.ctas, p.threads, p.smem, s>>>(p.d_desc, p.d_begin, p.n,
                                                                     b->roots);
    PK_CHECK_LAUNCH("batch_ntt_pass_kernel");
  }
  batch_leaves_kernel<<<(int)std::max<uint64_t>(1, std::min<uint64_t>((b->leaves.total + 127) / 128,
                                                                     (uint64_t)sm_count() * 64)),
                        128, 0, s>>>(b->leaves.d_desc, b->leaves.d_begin, b->leaves.n,
                                     b->leaves.total);
  PK_CHECK_LAUNCH("batch_leaves_kernel");
  for (auto& l : b->levels) {
    batch_level_kernel<<<(int)std::max<uint64_t>(1, std::min<uint64_t>((l.total + 127) / 128,
                                                                      (uint64_t)sm_count() * 64)),
                         128, 0, s>>>(l.d_desc, l.d_begin, l.n, l.total);
    PK_CHECK_LAUNCH("batch_level_kernel");
  }
  // sumcheck
  batch_copy_kernel<<<ew_blocks(b->copy_sc.total), 256, 0, s>>>(b->copy_sc.d_desc, b->copy_sc.d_begin,
                                                                b->copy_sc.n, b->copy_sc.total);
  PK_CHECK_LAUNCH("batch_copy_kernel");
  const int jb_blocks = (int)((nj + 63) / 64);
  batch_sc_start_kernel<<<jb_blocks, 64, 0, s>>>(b->d_state, b->d_jobs, nj);
  PK_CHECK_LAUNCH("batch_sc_start_kernel");
  batch_eq_half_kernel<<<ew_blocks(b->eq_half.total), 256, 0, s>>>(
      b->eq_half.d_desc, b->eq_half.d_begin, b->eq_half.n, b->eq_half.total, b->d_state, b->d_jobs);
  PK_CHECK_LAUNCH("batch_eq_half_kernel");
  batch_eq_combine_kernel<<<ew_blocks(b->eq_comb.total), 256, 0, s>>>(
      b->eq_comb.d_desc, b->eq_comb.d_begin, b->eq_comb.n, b->eq_comb.total, b->d_jobs);
  PK_CHECK_LAUNCH("batch_eq_combine_kernel");
  for (uint32_t r = 0; r < b->max_m0; r++) {
    const Grouped& g = b->rounds[r];
    if (r == 0)
      batch_sc_round_kernel<false><<<(unsigned)g.total, kScThreads, 0, s>>>(
          g.d_desc, g.d_begin, g.n, b->d_jobs, b->d_state, r);
    else
      batch_sc_round_kernel<true><<<(unsigned)g.total, kScThreads, 0, s>>>(
          g.d_desc, g.d_begin, g.n, b->d_jobs, b->d_state, r);
    PK_CHECK_LAUNCH("batch_sc_round_kernel");
    batch_sc_finish_round_kernel<<<jb_blocks, 64, 0, s>>>(b->d_state, b->d_jobs, nj, r,
                                                          b->d_nctas + (size_t)r * nj);
    PK_CHECK_LAUNCH("batch_sc_finish_round_kernel");
  }
  batch_sc_end_kernel<<<jb_blocks, 64, 0, s>>>(b->d_state, nj);
  PK_CHECK_LAUNCH("batch_sc_end_kernel");
  return PKG_OK;
}

static void drop_graph(pkg_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

static int batch_replan(pkg_batch* b) {
  drop_graph(b);
  int rc = batch_plan(b);
  if (rc) return rc;
  const size_t nj = b->jobs.size();
  std::vector<uint32_t> nctas(b->round_ctas.size());
  for (size_t i = 0; i < nctas.size(); i++) nctas[i] = (uint32_t)b->round_ctas[i];
  if (b->d_nctas) cudaFree(b->d_nctas);
  b->d_nctas = nullptr;
  PK_CUDA(cudaMalloc(&b->d_nctas, 4 * std::max<size_t>(nctas.size(), 1)));
  if (!nctas.empty())
    PK_CUDA(cudaMemcpy(b->d_nctas, nctas.data(), 4 * nctas.size(), cudaMemcpyHostToDevice));
  (void)nj;
  return PKG_OK;
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_batch_create(const uint32_t* log_sizes, size_t njobs, uint64_t seed,
                                pkg_batch** out) {
  PK_REQUIRE(out && (njobs == 0 || log_sizes), "null pointer");
  PK_REQUIRE(njobs >= 1 && njobs <= 4096, "njobs %zu out of range [1, 4096]", njobs);
  for (size_t j = 0; j < njobs; j++)
    PK_REQUIRE(log_sizes[j] >= 4 && log_sizes[j] <= 24, "job %zu: log size %u out of [4, 24]", j,
               log_sizes[j]);
  pkg_batch* b = new pkg_batch();
  b->log_n.assign(log_sizes, log_sizes + njobs);
  // sizes
  size_t bytes = 0;
  std::vector<size_t> offs(njobs);
  size_t max_order = 1024;
  for (size_t j = 0; j < njobs; j++) {
    const size_t n = size_t(1) << log_sizes[j];
    const size_t cw_rows = n / 2;  // (n / 8 messages) * 4
    const int m0 = (int)log_sizes[j];
    const int nhi = (m0 + 1) / 2, nlo = m0 - nhi;
    offs[j] = bytes;
    bytes += align256(32 * n) * 2;                         // coeffs, ntt
    bytes += align256(32 * 4 * n);                         // codeword
    bytes += align256(32 * (2 * cw_rows - 1));             // layers
    bytes += align256(32 * n) * 4;                         // a, b, c, eq
    bytes += align256(32 * (size_t(1) << nhi)) + align256(32 * (size_t(1) << nlo));
    bytes += align256(32 * 3 * kScCtaCap);                 // partials
    max_order = std::max(max_order, n);
  }
  cudaError_t e = cudaMalloc(&b->arena, bytes);
  if (e != cudaSuccess) {
    delete b;
    return cuda_status(e, "pkg_batch_create arena");
  }
  b->jobs.resize(njobs);
  b->init_state.resize(njobs);
  for (size_t j = 0; j < njobs; j++) {
    const size_t n = size_t(1) << log_sizes[j];
    JobDev& jb = b->jobs[j];
    uint8_t* p = b->arena + offs[j];
    auto take = [&](size_t nbytes) {
      uint8_t* q = p;
      p += align256(nbytes);
      return q;
    };
    jb.n = n;
    jb.log_n = log_sizes[j];
    jb.cw_rows = n / 2;
    jb.m0 = log_sizes[j];
    jb.nhi = (jb.m0 + 1) / 2;
    jb.nlo = jb.m0 - jb.nhi;
    jb.coeffs = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.ntt = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.cw = reinterpret_cast<uint64_t*>(take(32 * 4 * n));
    jb.layers = take(32 * (2 * jb.cw_rows - 1));
    jb.a = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.b = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.c = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.eq = reinterpret_cast<uint64_t*>(take(32 * n));
    jb.eq_hi = reinterpret_cast<uint64_t*>(take(32 * (size_t(1) << jb.nhi)));
    jb.eq_lo = reinterpret_cast<uint64_t*>(take(32 * (size_t(1) << jb.nlo)));
    jb.part = reinterpret_cast<uint64_t*>(take(32 * 3 * kScCtaCap));
    // sumcheck state: blinding g and w1 blinding values from the sampler
    ScState& st = b->init_state[j];
    memset(&st, 0, sizeof st);
    st.m0 = jb.m0;
    std::vector<uint64_t> g(16 * jb.m0), wb(16 * jb.m0);
    pkg_sample_fr(seed + 0x100000 + j, 4 * jb.m0, g.data(), 1);
    pkg_sample_fr(seed + 0x200000 + j, 4 * jb.m0, wb.data(), 1);
    memcpy(st.g, g.data(), 32 * 4 * jb.m0);
    memcpy(st.wb, wb.data(), 32 * 4 * jb.m0);
    uint64_t dom[4] = {j + 1, 0, 0, 0};
    memcpy(st.domain.v, dom, 32);
  }
  // inputs: job j's coefficients from pkg_sample_fr(seed + j); jobs are
  // sampled on all host threads (each job is its own ChaCha stream)
  {
    const unsigned nthreads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::atomic<size_t> next{0};
    std::atomic<int> failed{0};
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthreads; t++)
      pool.emplace_back([&, dev]() {
        if (cudaSetDevice(dev) != cudaSuccess) failed = 1;
        std::vector<uint64_t> host;
        for (size_t j = next++; j < njobs; j = next++) {
          const size_t n = b->jobs[j].n;
          host.resize(4 * n);
          pkg_sample_fr(seed + j, n, host.data(), 1);
          if (cudaMemcpy(b->jobs[j].coeffs, host.data(), 32 * n, cudaMemcpyHostToDevice) !=
              cudaSuccess)
            failed = 1;
        }
      });
    for (auto& th : pool) th.join();
    if (failed) {
      pkg_batch_destroy(b);
      set_last_error("pkg_batch_create: input upload failed");
      return PKG_ERR_CUDA;
    }
  }
  e = cudaMalloc(&b->d_jobs, sizeof(JobDev) * njobs);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_state, sizeof(ScState) * njobs);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_state_init, sizeof(ScState) * njobs);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_state_init, b->init_state.data(), sizeof(ScState) * njobs,
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_jobs, b->jobs.data(), sizeof(JobDev) * njobs, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    pkg_batch_destroy(b);
    return cuda_status(e, "pkg_batch_create tables");
  }
  int rc = roots_reserve(max_order, &b->roots);
  if (!rc) rc = batch_replan(b);
  if (rc) {
    pkg_batch_destroy(b);
    return rc;
  }
  *out = b;
  return PKG_OK;
}

extern "C" void pkg_batch_destroy(pkg_batch* b) {
  if (!b) return;
  drop_graph(b);
  cudaFree(b->arena);
  cudaFree(b->d_jobs);
  cudaFree(b->d_state);
  cudaFree(b->d_state_init);
  cudaFree(b->d_nctas);
  cudaFree(b->tables);
  delete b;
}

extern "C" int pkg_batch_job_info(pkg_batch* b, size_t j, pkg_batch_job* out) {
  PK_REQUIRE(b && out && j < b->jobs.size(), "bad batch/job");
  const JobDev& jb = b->jobs[j];
  out->log_n = jb.log_n;
  out->n = jb.n;
  out->coeffs = jb.coeffs;
  out->ntt = jb.ntt;
  out->codeword = jb.cw;
  out->layers = jb.layers;
  out->num_leaves = jb.cw_rows;
  out->transcript_domain = j + 1;
  const ScState& st = b->init_state[j];
  static_assert(sizeof(out->g) == sizeof(st.g) && sizeof(out->w1_blinding) == sizeof(st.wb),
                "job info mirrors the sumcheck state");
  memcpy(out->g, st.g, sizeof out->g);
  memcpy(out->w1_blinding, st.wb, sizeof out->w1_blinding);
  return PKG_OK;
}

extern "C" int pkg_batch_set_params(pkg_batch* b, int kmax, int log_elems_per_cta) {
  PK_REQUIRE(b, "null batch");
  PK_REQUIRE(kmax >= 1 && kmax <= 11, "kmax %d out of [1, 11]", kmax);
  PK_REQUIRE(log_elems_per_cta >= kmax && log_elems_per_cta <= 11,
             "elements per CTA 2^%d must be in [2^kmax, 2^11]", log_elems_per_cta);
  b->kmax = kmax;
  b->log_elems = log_elems_per_cta;
  return batch_replan(b);
}

extern "C" int pkg_batch_set_butterflies_per_thread(pkg_batch* b, int log_bpt) {
  PK_REQUIRE(b, "null batch");
  PK_REQUIRE(log_bpt >= 0 && log_bpt <= 2, "butterflies per thread 2^%d out of [1, 4]", log_bpt);
  b->log_bpt = log_bpt;
  return batch_replan(b);
}

extern "C" int pkg_batch_get_params(pkg_batch* b, int* kmax, int* log_elems_per_cta,
                                    int* log_butterflies_per_thread) {
  PK_REQUIRE(b, "null batch");
  if (kmax) *kmax = b->kmax;
  if (log_elems_per_cta) *log_elems_per_cta = b->log_elems;
  if (log_butterflies_per_thread) *log_butterflies_per_thread = b->log_bpt;
  return PKG_OK;
}

extern "C" int pkg_batch_run(pkg_batch* b, int use_graph, pkg_stream_t stream) {
  PK_REQUIRE(b, "null batch");
  cudaStream_t s = as_stream(stream);
  if (!use_graph) return batch_enqueue(b, s);
  if (!b->exec) {
    PK_REQUIRE(s != nullptr, "graph capture needs a non-default stream");
    PK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = pkg_kernel_launches();
    int rc = batch_enqueue(b, s);
    b->graph_kernels = pkg_kernel_launches() - before;
    count_launches_undo(b->graph_kernels);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    b->graph = g;
    PK_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  }
  PK_CUDA(cudaGraphLaunch(b->exec, s));
  count_launches_undo(0 - b->graph_kernels);  // the replay runs every captured kernel
  return PKG_OK;
}

extern "C" int pkg_batch_sumcheck_result(pkg_batch* b, size_t j, pkg_sumcheck_result* out) {
  PK_REQUIRE(b && out && j < b->jobs.size(), "bad batch/job");
  ScState st;
  PK_CUDA(cudaMemcpy(&st, b->d_state + j, sizeof st, cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof *out);
  out->m0 = st.m0;
  for (uint32_t i = 0; i < st.m0; i++) {
    memcpy(out->r[i], st.r[i].v, 32);
    memcpy(out->alpha[i], st.alpha[i].v, 32);
    for (int k = 0; k < 4; k++) memcpy(out->coeffs[4 * i + k], st.coeffs[i][k].v, 32);
  }
  memcpy(out->rho, st.rho.v, 32);
  memcpy(out->sum_g, st.sum_g.v, 32);
  memcpy(out->blinding_eval, st.blinding_eval.v, 32);
  memcpy(out->transcript.l, st.tl.v, 32);
  memcpy(out->transcript.r, st.tr.v, 32);
  return PKG_OK;
}

extern "C" int pkg_batch_tune(pkg_batch* b, pkg_stream_t stream, int* best_kmax,
                              int* best_log_elems, double* best_ms) {
  PK_REQUIRE(b, "null batch");
  cudaStream_t s = as_stream(stream);
  cudaEvent_t e0, e1;
  PK_CUDA(cudaEventCreate(&e0));
  PK_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int bk = b->kmax, be = b->log_elems, bb = b->log_bpt;
  for (int k = 4; k <= 11; k++) {
    for (int le = std::max(k, 8); le <= 11; le++) {
      for (int lb = 0; lb <= 2; lb++) {
        b->log_bpt = lb;
        int rc = pkg_batch_set_params(b, k, le);
        if (rc) return rc;
        if ((rc = batch_enqueue(b, s))) return rc;  // warm-up
        PK_CUDA(cudaEventRecord(e0, s));
        if ((rc = batch_enqueue(b, s))) return rc;
        PK_CUDA(cudaEventRecord(e1, s));
        PK_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          bk = k;
          be = le;
          bb = lb;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->log_bpt = bb;
  int rc = pkg_batch_set_params(b, bk, be);
  if (rc) return rc;
  if (best_kmax) *best_kmax = bk;
  if (best_log_elems) *best_log_elems = be;
  if (best_ms) *best_ms = best;
  return PKG_OK;
}
