// server.cu -- the served form: a request loop that admits proving jobs of
// different circuit sizes by their HBM footprint, keeps each job's R1CS,
// witness, codeword, Merkle layers and sumcheck tables resident on the
// device for the whole prove, and overlaps admitted jobs on the device (one
// worker thread + CUDA stream per in-flight slot).  Latencies (submit ->
// done) feed p50 / p99 / p99.9 and proofs/s.
//
// Admission: a queued request is admitted when the reserved footprint plus
// its estimate fits the budget and a slot is free.  Requests are considered
// first-fit in arrival order (a small request may pass a large one that does
// not fit yet), except that a request passed over 8 times blocks the queue
// until it fits, so large requests are not starved.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ntt_internal.cuh"
#include "host_stage.cuh"
#include "pk_common.cuh"

namespace pk {

static uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct HostRequest {
  uint64_t id = 0;
  size_t nc = 0, nw = 0, nnz[3] = {0, 0, 0};
  // the caller's buffers (valid until pkg_server_wait returns for this id)
  const uint64_t* row_ptr[3] = {nullptr, nullptr, nullptr};
  const uint32_t* cols[3] = {nullptr, nullptr, nullptr};
  const uint64_t* vals[3] = {nullptr, nullptr, nullptr};
  const uint64_t* witness = nullptr;
  size_t num_public = 0;
  uint64_t blinding_seed = 0, domain = 0;
  unsigned ff = 3, lr = 2;
  // whole proof: WHIR parameters and the caller's output buffers
  bool whole = false;
  pkg_whir_params whir{};
  uint64_t* whir_commit_words = nullptr;
  uint64_t* whir_proof = nullptr;
  size_t footprint = 0;
  int passed_over = 0;
  // results
  uint64_t t_submit = 0, t_admit = 0, t_done = 0;
  int status = 1;  // 1 = pending, 0 = ok, < 0 = error
  std::string error;
  pkg_spartan_proof proof;
};

static size_t ceil_log2_sz(size_t n) {
  size_t p = 1, k = 0;
  while (p < n) {
    p <<= 1;
    k++;
  }
  return k;
}

// Device bytes pkg_spartan_prove (with whole, pkg_prove_r1cs) plus the
// resident request use (upper bound).
size_t prove_footprint(size_t nc, size_t nw, const size_t nnz[3], unsigned ff, unsigned lr,
                       bool whole, unsigned batch) {
  size_t m = ceil_log2_sz(nw), m0 = ceil_log2_sz(nc);
  if (m < 13) m = 13;
  if (m0 < 1) m0 = 1;
  if ((size_t(1) << m) - nw < 4 * m0) m++;
  const size_t n = size_t(1) << m, cw = n << lr, L = cw >> ff;
  size_t b = 0;
  b += 32 * n;                      // padded witness polynomial
  b += 32 * cw;                     // codeword
  b += 32 * (2 * L);                // Merkle layers
  b += 32 * 3 * (size_t(1) << m0);  // sumcheck tables
  b += 32 * (size_t(1) << m0);      // eq(r)
  b += 32 * (nc + nw);              // eq(alpha), alpha covector
  size_t maxnnz = std::max(nnz[0], std::max(nnz[1], nnz[2]));
  b += 8 * (nw + 1) + 36 * maxnnz + (4 << 20);  // one transposed matrix + scan temp
  for (int k = 0; k < 3; k++) b += 8 * (nc + 1) + 36 * nnz[k];  // resident R1CS
  b += 32 * nw;                                                   // resident witness
  if (whole) {
    // the WHIR rounds: up to five padded statement covectors (public
    // weight, A, B, C, blinding), f^ and w tables, two folded polynomials,
    // and two round codewords with their trees at a time (the first
    // round's, the largest, holds n << (lr - 1) Fr)
    const size_t cw1 = lr >= 1 ? n << (lr - 1) : n;
    b += 32 * 5 * n + 32 * 2 * n + 32 * 2 * (n >> ff);
    b += 2 * (32 * cw1 + 32 * 2 * (cw1 >> ff));
    // whir-ZK: the blinding polynomial, the second half of the first
    // codeword, and the batch's combination
    b += (size_t)(batch - 1) * (32 * n + 32 * cw + 32 * n);
  }
  return b + b / 8 + (16 << 20);                                  // pool slack
}

}  // namespace pk

struct pkg_server {
  int device = 0;
  size_t budget = 0, reserved = 0, peak_reserved = 0;
  int slots = 1, inflight = 0;
  bool stopping = false;
  uint64_t next_id = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<pk::HostRequest>> queue;      // waiting for admission
  std::deque<std::shared_ptr<pk::HostRequest>> admitted;   // admitted, not yet picked
  std::map<uint64_t, std::shared_ptr<pk::HostRequest>> all;
  std::vector<std::thread> workers;
  std::vector<uint64_t> latencies_ns;
  uint64_t first_submit = 0, last_done = 0;
};

namespace pk {

// Move every admissible request from queue to admitted (caller holds mu).
static void admit_locked(pkg_server* s) {
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    if (s->inflight + (int)s->admitted.size() >= s->slots) break;
    auto& r = *it;
    if (s->reserved + r->footprint <= s->budget) {
      s->reserved += r->footprint;
      s->peak_reserved = std::max(s->peak_reserved, s->reserved);
      r->t_admit = now_ns();
      s->admitted.push_back(r);
      it = s->queue.erase(it);
      s->cv_work.notify_one();
      continue;
    }
    if (++r->passed_over > 8) break;  // hold the queue for a starved request
    ++it;
  }
}

static int run_request(HostRequest& r, cudaStream_t st) {
  std::vector<void*> bufs;
  cudaMemPool_t pool = lib_pool();
  if (!pool) return PKG_ERR_CUDA;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 256), pool, st) != cudaSuccess)
      return nullptr;
    bufs.push_back(p);
    return p;
  };
  pkg_r1cs rc1;
  memset(&rc1, 0, sizeof rc1);
  rc1.num_constraints = r.nc;
  rc1.num_witnesses = r.nw;
  rc1.num_public_inputs = r.num_public;
  int rc = PKG_OK;
  // (destination, host source, bytes) of every upload
  struct Up {
    void* dst;
    const void* src;
    size_t bytes;
  };
  std::vector<Up> ups;
  for (int k = 0; k < 3 && !rc; k++) {
    void* rp = alloc(8 * (r.nc + 1));
    void* cl = alloc(4 * r.nnz[k]);
    void* vl = alloc(32 * r.nnz[k]);
    if (!rp || !cl || !vl) {
      rc = PKG_ERR_OUT_OF_MEMORY;
      break;
    }
    ups.push_back({rp, r.row_ptr[k], 8 * (r.nc + 1)});
    if (r.nnz[k]) {
      ups.push_back({cl, r.cols[k], 4 * r.nnz[k]});
      ups.push_back({vl, r.vals[k], 32 * r.nnz[k]});
    }
    rc1.row_ptr[k] = static_cast<uint64_t*>(rp);
    rc1.cols[k] = static_cast<uint32_t*>(cl);
    rc1.vals[k] = static_cast<uint64_t*>(vl);
    rc1.nnz[k] = r.nnz[k];
  }
  void* w = rc ? nullptr : alloc(32 * r.nw);
  if (!rc && !w) rc = PKG_ERR_OUT_OF_MEMORY;
  if (!rc) {
    ups.push_back({w, r.witness, 32 * r.nw});
    // Uploads go through the host stager (pinned chunks, threaded host copies)
    // rather than pageable copies from several workers at once; the worker's
    // stream waits for them.  The buffers were allocated on `st`, so the
    // stager's stream first waits for `st`.
    HostStager& hs = HostStager::current();
    std::lock_guard<std::mutex> lk(hs.mutex());
    rc = hs.ensure();
    cudaEvent_t allocated = nullptr;
    if (!rc && cudaEventCreateWithFlags(&allocated, cudaEventDisableTiming) != cudaSuccess)
      rc = PKG_ERR_CUDA;
    if (!rc && (cudaEventRecord(allocated, st) != cudaSuccess ||
                cudaStreamWaitEvent(hs.stream(), allocated, 0) != cudaSuccess))
      rc = PKG_ERR_CUDA;
    for (size_t i = 0; !rc && i < ups.size(); i++)
      rc = hs.h2d(static_cast<uint8_t*>(ups[i].dst), ups[i].src, ups[i].bytes);
    if (!rc) rc = hs.handoff(st);
    if (allocated) cudaEventDestroy(allocated);
  }
  if (!rc) {
    rc = r.whole ? pkg_prove_r1cs(&rc1, static_cast<uint64_t*>(w), r.blinding_seed, r.domain,
                                  &r.whir, &r.proof, r.whir_commit_words, r.whir_proof, st)
                 : pkg_spartan_prove(&rc1, static_cast<uint64_t*>(w), r.blinding_seed, r.domain,
                                     r.ff, r.lr, &r.proof, st);
    if (rc) r.error = pkg_last_error();
  } else if (r.error.empty()) {
    r.error = pkg_last_error();
  }
  for (void* p : bufs) cudaFreeAsync(p, st);
  cudaStreamSynchronize(st);
  return rc;
}

// Pinned staging each worker allocates at start: a whole proof's STIR
// openings at 2^22 constraints take ~0.4 MB.
constexpr size_t kWorkerStageBytes = size_t(1) << 20;

static void worker_main(pkg_server* s) {
  cudaSetDevice(s->device);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  // the worker's per-thread buffers before its first request, not inside it
  // (a failure here only leaves them to the first request)
  if (warm_thread_resources(kWorkerStageBytes)) cudaGetLastError();
  for (;;) {
    std::shared_ptr<HostRequest> r;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stopping || !s->admitted.empty(); });
      if (s->admitted.empty()) break;  // stopping and drained
      r = s->admitted.front();
      s->admitted.pop_front();
      s->inflight++;
    }
    int rc = run_request(*r, st);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->t_done = now_ns();
      r->status = rc;
      s->inflight--;
      s->reserved -= r->footprint;
      if (rc == PKG_OK) {
        s->latencies_ns.push_back(r->t_done - r->t_submit);
        s->last_done = std::max(s->last_done, r->t_done);
      }
      admit_locked(s);
    }
    s->cv_done.notify_all();
  }
  cudaStreamDestroy(st);
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_server_create(size_t hbm_budget_bytes, int max_inflight, pkg_server** out) {
  PK_REQUIRE(out, "null output");
  PK_REQUIRE(max_inflight >= 1 && max_inflight <= 64, "max_inflight %d out of [1, 64]",
             max_inflight);
  size_t free_b = 0, total_b = 0;
  PK_CUDA(cudaMemGetInfo(&free_b, &total_b));
  // memory the library pool holds but does not use is available as well
  PK_REQUIRE(lib_pool() != nullptr, "could not create the library memory pool");
  uint64_t reserved = 0, used = 0;
  PK_CUDA(cudaMemPoolGetAttribute(lib_pool(), cudaMemPoolAttrReservedMemCurrent, &reserved));
  PK_CUDA(cudaMemPoolGetAttribute(lib_pool(), cudaMemPoolAttrUsedMemCurrent, &used));
  const size_t avail = free_b + (size_t)(reserved > used ? reserved - used : 0);
  PK_REQUIRE(hbm_budget_bytes > 0 && hbm_budget_bytes <= avail,
             "budget %zu bytes exceeds available device memory %zu", hbm_budget_bytes, avail);
  // Twiddles for every transform the admitted sizes can need (codewords up to
  // 2^28): built once here, before any worker runs.
  const uint64_t* roots = nullptr;
  int rc = roots_reserve(size_t(1) << 24, &roots);
  if (rc) return rc;
  // Request buffers come from the library's pool, which keeps freed memory,
  // so back-to-back proves reuse it instead of mapping it again.  The budget
  // is reserved in the pool once, here: allocated and freed on a private
  // stream and waited for, so every later request, on any worker stream, is
  // carved from memory whose free has completed -- the pool neither grows
  // (a physical mapping in the middle of a request) nor chains the workers'
  // streams while requests run.
  if ((rc = pkg_reserve_memory(hbm_budget_bytes))) return rc;
  pkg_server* s = new pkg_server();
  PK_CUDA(cudaGetDevice(&s->device));
  s->budget = hbm_budget_bytes;
  s->slots = max_inflight;
  for (int i = 0; i < max_inflight; i++) s->workers.emplace_back(worker_main, s);
  *out = s;
  return PKG_OK;
}

extern "C" int pkg_server_submit(pkg_server* s, const pkg_prove_request* req, uint64_t* id_out) {
  PK_REQUIRE(s && req && id_out, "null pointer");
  PK_REQUIRE(req->num_constraints >= 1 && req->num_witnesses >= 1 && req->witness,
             "empty request");
  auto r = std::make_shared<HostRequest>();
  r->nc = req->num_constraints;
  r->nw = req->num_witnesses;
  for (int k = 0; k < 3; k++) {
    PK_REQUIRE(req->row_ptr[k] && (req->nnz[k] == 0 || (req->cols[k] && req->vals[k])),
               "null matrix array");
    // the row pointers bound every device walk over a row's entries: they
    // start at 0, never decrease and end at nnz (column indices are checked
    // on the device, where an out-of-range one is skipped and reported)
    const uint64_t* rp = req->row_ptr[k];
    PK_REQUIRE(rp[0] == 0 && rp[r->nc] == req->nnz[k],
               "matrix %d: row pointers run from %llu to %llu, nnz is %zu", k,
               (unsigned long long)rp[0], (unsigned long long)rp[r->nc], req->nnz[k]);
    bool monotone = true;
    for (size_t i = 0; i < r->nc; i++) monotone &= rp[i + 1] >= rp[i];
    PK_REQUIRE(monotone, "matrix %d: row pointers decrease", k);
    r->nnz[k] = req->nnz[k];
    r->row_ptr[k] = req->row_ptr[k];
    r->cols[k] = req->cols[k];
    r->vals[k] = req->vals[k];
  }
  r->witness = req->witness;
  r->num_public = req->num_public_inputs;
  PK_REQUIRE(r->num_public + 1 <= r->nw, "%zu public inputs but %zu witnesses", r->num_public,
             r->nw);
  r->blinding_seed = req->blinding_seed;
  r->domain = req->transcript_domain;
  r->ff = req->folding_factor;
  r->lr = req->log_inv_rate;
  if (req->whir) {
    PK_REQUIRE(req->whir_commit_words && req->whir_proof, "null WHIR output buffer");
    PK_REQUIRE(pkg_whir_proof_words(req->whir, 3) != 0, "invalid WHIR parameters");
    size_t m = 0, m0 = 0;
    int rc = pkg_r1cs_sizing(r->nc, r->nw, &m, &m0);
    if (rc) return rc;
    PK_REQUIRE(req->whir->num_variables == m,
               "WHIR parameters for %u variables, the R1CS needs %zu", req->whir->num_variables,
               m);
    r->whole = true;
    r->whir = *req->whir;
    r->whir_commit_words = req->whir_commit_words;
    r->whir_proof = req->whir_proof;
    r->ff = r->whir.folding_factor;
    r->lr = r->whir.log_inv_rate;
  }
  r->footprint = prove_footprint(r->nc, r->nw, r->nnz, r->ff, r->lr, r->whole,
                                 r->whole ? r->whir.batch_size : 1);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->footprint > s->budget) {
      set_last_error("request needs ~%zu bytes, above the %zu-byte budget", r->footprint,
                     s->budget);
      return PKG_ERR_OUT_OF_MEMORY;
    }
    r->id = s->next_id++;
    r->t_submit = now_ns();
    if (!s->first_submit) s->first_submit = r->t_submit;
    s->all[r->id] = r;
    s->queue.push_back(r);
    admit_locked(s);
  }
  *id_out = r->id;
  return PKG_OK;
}

extern "C" int pkg_server_wait(pkg_server* s, uint64_t id, pkg_spartan_proof* proof,
                               pkg_request_times* times) {
  PK_REQUIRE(s, "null server");
  std::shared_ptr<HostRequest> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    PK_REQUIRE(it != s->all.end(), "unknown request id %llu", (unsigned long long)id);
    r = it->second;
    s->cv_done.wait(lk, [&] { return r->status != 1; });
    s->all.erase(id);
  }
  if (times) {
    times->submit_ns = r->t_submit;
    times->admit_ns = r->t_admit;
    times->done_ns = r->t_done;
    times->footprint_bytes = r->footprint;
  }
  if (r->status != PKG_OK) {
    set_last_error("request %llu failed: %s", (unsigned long long)id, r->error.c_str());
    return r->status;
  }
  if (proof) *proof = r->proof;
  return PKG_OK;
}

extern "C" int pkg_server_get_stats(pkg_server* s, pkg_server_stats* out) {
  PK_REQUIRE(s && out, "null pointer");
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof *out);
  std::vector<uint64_t> l = s->latencies_ns;
  out->completed = l.size();
  out->queued = s->queue.size() + s->admitted.size();
  out->inflight = s->inflight;
  out->reserved_bytes = s->reserved;
  out->peak_reserved_bytes = s->peak_reserved;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
      size_t i = (size_t)std::min<double>(l.size() - 1, std::ceil(p * l.size()) - 1);
      return l[i] * 1e-6;
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->p999_ms = pct(0.999);
    if (s->last_done > s->first_submit)
      out->proofs_per_s = l.size() / ((s->last_done - s->first_submit) * 1e-9);
  }
  return PKG_OK;
}

extern "C" void pkg_server_destroy(pkg_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (auto& r : s->queue) {  // not yet admitted: fail them so waiters return
      r->status = PKG_ERR_UNSUPPORTED;
      r->error = "server stopped before admission";
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->workers) t.join();
  delete s;
}
