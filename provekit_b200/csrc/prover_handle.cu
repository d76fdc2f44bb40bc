// prover_handle.cu -- the handle surface of the reference's C FFI
// (tooling/provekit-ffi/src/ffi.rs, types.rs) over the device prover:
//
//   pkg_prover           PKProver: a prepared circuit, here resident on one
//                        device with its transposes, plus the proof
//                        configuration; freed once by pkg_prover_free
//   pkg_prover_prove     pk_prove_json / pk_prove_toml (ffi.rs:537-666): a
//                        solved witness in, a library-owned proof buffer out
//   pkg_buf / pkg_free_buf   PKBuf (types.rs:8-40) and pk_free_buf (ffi.rs:744-750)
//   pkg_prover_serialize / pkg_prover_load_bytes
//                        pk_serialize_prover / pk_load_prover_bytes
//                        (ffi.rs:329-362, 455-482) over this library's own
//                        byte layout (the .pkp layout is postcard over the
//                        un-vendored whir / spongefish types)
//   pkg_get_last_error   pk_get_last_error (ffi.rs:73-89): take and clear
//   pkg_init             pk_init (ffi.rs:92-97)
//
// Conventions kept from the reference: int statuses, a thread-local message,
// no exception crosses the ABI, out parameters are reset on entry, buffers
// are freed exactly once by the library.  Every host input is validated on
// the host before any device work (row pointers, column indices, sizes), so
// a malformed circuit or byte string is an error status, never a device
// fault.
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "fr_host.hpp"
#include "host_stage.cuh"
#include "pk_common.cuh"

struct pkg_prover {
  int device = 0;
  std::mutex mu;  // one proof at a time per handle (its stream and witness buffer)
  size_t nc = 0, nw = 0, npub = 0, nnz[3] = {0, 0, 0};
  pkg_prover_config cfg{};
  pkg_whir_params whir{};
  size_t m = 0, m0 = 0;
  void* mats = nullptr;        // A, B, C in CSR (device)
  void* transposes = nullptr;  // their transposes (device)
  uint64_t* witness = nullptr; // one proof's witness (device)
  pkg_r1cs r1cs{};             // device view of the above
  cudaStream_t stream = nullptr;
};

namespace pk {
namespace {

constexpr char kProofMagic[8] = {'P', 'K', 'G', 'P', 'R', 'O', 'O', 'F'};
constexpr char kProverMagic[8] = {'P', 'K', 'G', 'P', 'R', 'O', 'V', 'R'};
constexpr uint32_t kFormatVersion = 1;

size_t align_up(size_t b, size_t a) { return (b + a - 1) / a * a; }

// The device switch of one entry point, undone on return.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void free_handle(pkg_prover* p) {
  if (!p) return;
  DeviceScope ds(p->device);
  if (p->stream) {
    cudaStreamSynchronize(p->stream);
    cudaStreamDestroy(p->stream);
  }
  if (p->witness) cudaFree(p->witness);
  if (p->transposes) cudaFree(p->transposes);
  if (p->mats) cudaFree(p->mats);
  cudaGetLastError();
  delete p;
}

// CSR checks the device kernels rely on: row pointers start at 0, never
// decrease and end at nnz; every column is a witness index; every
// coefficient is a canonical field element (below p, as ark-ff's validating
// deserialisation requires and the device arithmetic assumes).
int check_csr(int k, size_t rows, size_t cols, const uint64_t* rp, const uint32_t* cl,
              const uint64_t* vl, size_t nnz) {
  PK_REQUIRE(rp, "matrix %d: null row pointers", k);
  PK_REQUIRE(nnz == 0 || cl, "matrix %d: null columns", k);
  PK_REQUIRE(rp[0] == 0, "matrix %d: row pointers must start at 0", k);
  for (size_t i = 0; i < rows; i++)
    PK_REQUIRE(rp[i + 1] >= rp[i], "matrix %d: row pointer %zu decreases", k, i + 1);
  PK_REQUIRE(rp[rows] == nnz, "matrix %d: row pointers end at %llu, nnz is %zu", k,
             (unsigned long long)rp[rows], nnz);
  for (size_t e = 0; e < nnz; e++)
    PK_REQUIRE(cl[e] < cols, "matrix %d: column %u of entry %zu is not a witness index (< %zu)",
               k, cl[e], e, cols);
  for (size_t e = 0; e < nnz; e++)
    PK_REQUIRE(HostFr::from_limbs(vl + 4 * e).is_canonical(),
               "matrix %d: coefficient %zu is not a canonical field element (>= p)", k, e);
  return PKG_OK;
}

int make_whir(const pkg_prover_config* cfg, size_t m, pkg_whir_params* out) {
  int rc = pkg_whir_params_init(out, (unsigned)m, cfg->folding_factor, cfg->log_inv_rate,
                                cfg->security_bits, cfg->pow_bits);
  if (rc) return rc;
  out->batch_size = cfg->zk ? 2 : 1;
  PK_REQUIRE(pkg_whir_proof_words(out, 5) != 0, "invalid WHIR parameters for m = %zu", m);
  return PKG_OK;
}

// Little-endian writer / reader of the byte layouts below.
struct Writer {
  uint8_t* at;
  void bytes(const void* p, size_t n) {
    memcpy(at, p, n);
    at += n;
  }
  void u32(uint32_t v) { bytes(&v, 4); }
  void u64(uint64_t v) { bytes(&v, 8); }
  void zeros(size_t n) {
    memset(at, 0, n);
    at += n;
  }
};

struct Reader {
  const uint8_t* at;
  const uint8_t* end;
  bool take(void* dst, size_t n) {
    if ((size_t)(end - at) < n) return false;
    memcpy(dst, at, n);
    at += n;
    return true;
  }
  bool skip(size_t n) {
    if ((size_t)(end - at) < n) return false;
    at += n;
    return true;
  }
};

// Fr in the Spartan part of a proof after the root: m0 challenges r, 4 m0
// round coefficients, m0 challenges alpha, rho, sum_g, blinding_eval,
// public_x, 3 evaluations, public_hash, public_eval, the transcript (2 Fr).
size_t spartan_fr(size_t m0) { return 6 * m0 + 11; }

// magic, version, reserved word, seven u64 fields
constexpr size_t kProofHeader = 8 + 4 + 4 + 7 * 8;

size_t proof_bytes(const pkg_prover* p, size_t nstm) {
  return kProofHeader + 104 + 32 + 32 * spartan_fr(p->m0) + 8 * pkg_whir_commit_words(&p->whir) +
         8 * pkg_whir_proof_words(&p->whir, nstm);
}

}  // namespace
}  // namespace pk

using namespace pk;

static_assert(sizeof(pkg_whir_params) == 104, "WHIR parameters are 26 u32 words");

extern "C" int pkg_init(void) {
  clear_last_error();
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return cuda_status(e, "pkg_init: cudaGetDeviceCount");
  if (n < 1) {
    set_last_error("pkg_init: no CUDA device");
    return PKG_ERR_CUDA;
  }
  return PKG_OK;
}

extern "C" int pkg_get_last_error(pkg_buf* out) {
  if (!out) return PKG_ERR_INVALID_ARGUMENT;
  *out = pkg_buf{nullptr, 0, 0};
  const char* msg = pkg_last_error();
  const size_t n = strlen(msg);
  if (n) {
    uint8_t* p = static_cast<uint8_t*>(malloc(n));
    if (!p) return PKG_ERR_OUT_OF_MEMORY;
    memcpy(p, msg, n);
    *out = pkg_buf{p, n, n};
  }
  clear_last_error();
  return PKG_OK;
}

extern "C" void pkg_free_buf(pkg_buf buf) {
  if (buf.ptr) free(buf.ptr);
}

extern "C" int pkg_prover_config_default(pkg_prover_config* cfg) {
  PK_REQUIRE(cfg, "null config");
  memset(cfg, 0, sizeof *cfg);
  // provekit/r1cs-compiler/src/whir_r1cs.rs:94-117 with WhirZkConfig
  cfg->folding_factor = 3;
  cfg->log_inv_rate = 2;
  cfg->security_bits = 128;
  cfg->pow_bits = 10;
  cfg->zk = 1;
  cfg->transcript_domain = 0;
  return PKG_OK;
}

extern "C" int pkg_prover_create(size_t num_constraints, size_t num_witnesses,
                                 size_t num_public_inputs, const uint64_t* const row_ptr[3],
                                 const uint32_t* const cols[3], const uint64_t* const vals[3],
                                 const size_t nnz[3], const pkg_prover_config* cfg,
                                 pkg_prover** out) {
  PK_REQUIRE(out, "null output");
  *out = nullptr;
  clear_last_error();
  PK_REQUIRE(row_ptr && cols && vals && nnz && cfg, "null pointer");
  PK_REQUIRE(num_constraints >= 1 && num_witnesses >= 1, "empty R1CS");
  PK_REQUIRE(num_witnesses < (size_t(1) << 32) && num_constraints < (size_t(1) << 32),
             "R1CS dimensions must fit u32 indices");
  PK_REQUIRE(num_public_inputs + 1 <= num_witnesses, "%zu public inputs but %zu witnesses",
             num_public_inputs, num_witnesses);
  size_t m = 0, m0 = 0;
  int rc = pkg_r1cs_sizing(num_constraints, num_witnesses, &m, &m0);
  if (rc) return rc;
  PK_REQUIRE(m <= 28 && m0 <= 30, "instance too large (m = %zu, m0 = %zu)", m, m0);
  for (int k = 0; k < 3; k++) {
    PK_REQUIRE(nnz[k] == 0 || vals[k], "matrix %d: null values", k);
    if ((rc = check_csr(k, num_constraints, num_witnesses, row_ptr[k], cols[k], vals[k],
                        nnz[k])))
      return rc;
  }
  pkg_whir_params whir;
  if ((rc = make_whir(cfg, m, &whir))) return rc;

  pkg_prover* p = new (std::nothrow) pkg_prover();
  if (!p) {
    set_last_error("out of host memory");
    return PKG_ERR_OUT_OF_MEMORY;
  }
  auto fail = [&](int code) {
    free_handle(p);
    return code;
  };
  {
    const cudaError_t e0 = cudaGetDevice(&p->device);
    if (e0 != cudaSuccess) return fail(cuda_status(e0, "pkg_prover_create: cudaGetDevice"));
  }
  p->nc = num_constraints;
  p->nw = num_witnesses;
  p->npub = num_public_inputs;
  p->cfg = *cfg;
  p->whir = whir;
  p->m = m;
  p->m0 = m0;
  // one device block for the three matrices, 256-byte aligned parts
  size_t off[3][3], total = 0;
  for (int k = 0; k < 3; k++) {
    p->nnz[k] = nnz[k];
    const size_t e = nnz[k] ? nnz[k] : 1;
    off[k][0] = total;
    total += align_up(8 * (num_constraints + 1), 256);
    off[k][1] = total;
    total += align_up(4 * e, 256);
    off[k][2] = total;
    total += align_up(32 * e, 256);
  }
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&p->mats, total);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->witness), 32 * num_witnesses);
  if (e != cudaSuccess) return fail(cuda_status(e, "pkg_prover_create: device memory"));
  uint8_t* base = static_cast<uint8_t*>(p->mats);
  p->r1cs.num_constraints = num_constraints;
  p->r1cs.num_witnesses = num_witnesses;
  p->r1cs.num_public_inputs = num_public_inputs;
  for (int k = 0; k < 3 && e == cudaSuccess; k++) {
    p->r1cs.row_ptr[k] = reinterpret_cast<uint64_t*>(base + off[k][0]);
    p->r1cs.cols[k] = reinterpret_cast<uint32_t*>(base + off[k][1]);
    p->r1cs.vals[k] = reinterpret_cast<uint64_t*>(base + off[k][2]);
    p->r1cs.nnz[k] = nnz[k];
    e = cudaMemcpy(base + off[k][0], row_ptr[k], 8 * (num_constraints + 1),
                   cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnz[k])
      e = cudaMemcpy(base + off[k][1], cols[k], 4 * nnz[k], cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnz[k])
      e = cudaMemcpy(base + off[k][2], vals[k], 32 * nnz[k], cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) return fail(cuda_status(e, "pkg_prover_create: upload"));
  // the transposes, once for the handle's life (transpose_r1cs_matrices,
  // provekit/common/src/utils/sumcheck.rs:195-206)
  e = cudaMalloc(&p->transposes, pkg_r1cs_transposes_bytes(&p->r1cs));
  if (e != cudaSuccess) return fail(cuda_status(e, "pkg_prover_create: transposes"));
  if ((rc = pkg_r1cs_build_transposes(&p->r1cs, p->transposes,
                                      reinterpret_cast<pkg_stream_t>(p->stream))))
    return fail(rc);
  e = cudaStreamSynchronize(p->stream);
  if (e != cudaSuccess) return fail(cuda_status(e, "pkg_prover_create"));
  *out = p;
  return PKG_OK;
}

extern "C" void pkg_prover_free(pkg_prover* prover) { free_handle(prover); }

extern "C" int pkg_prover_get_info(const pkg_prover* p, pkg_prover_info* info) {
  PK_REQUIRE(p && info, "null pointer");
  memset(info, 0, sizeof *info);
  info->num_constraints = p->nc;
  info->num_witnesses = p->nw;
  info->num_public_inputs = p->npub;
  info->m = p->m;
  info->m0 = p->m0;
  info->num_statements = 4 + (p->npub ? 1 : 0);
  info->proof_bytes = proof_bytes(p, info->num_statements);
  info->device = p->device;
  info->whir = p->whir;
  return PKG_OK;
}

extern "C" int pkg_prover_prove(pkg_prover* p, const uint64_t* witness, uint64_t blinding_seed,
                                pkg_buf* out_proof) {
  PK_REQUIRE(out_proof, "null output");
  *out_proof = pkg_buf{nullptr, 0, 0};
  clear_last_error();
  PK_REQUIRE(p && witness, "null pointer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceScope ds(p->device);
  PK_REQUIRE(ds.ok, "cannot select device %d", p->device);
  // a previous call that failed part-way may have left work reading the
  // witness buffer
  PK_CUDA(cudaStreamSynchronize(p->stream));
  const size_t nstm = 4 + (p->npub ? 1 : 0);
  const size_t bytes = proof_bytes(p, nstm);
  uint8_t* buf = static_cast<uint8_t*>(malloc(bytes));
  if (!buf) {
    set_last_error("out of host memory for a %zu-byte proof", bytes);
    return PKG_ERR_OUT_OF_MEMORY;
  }
  const size_t cwords = pkg_whir_commit_words(&p->whir);
  const size_t pwords = pkg_whir_proof_words(&p->whir, nstm);
  uint8_t* spartan_at = buf + kProofHeader + 104;
  uint64_t* commit_at = reinterpret_cast<uint64_t*>(spartan_at + 32 + 32 * spartan_fr(p->m0));
  uint64_t* proof_at = commit_at + cwords;
  // the witness through the host stager (pinned chunks, threaded host
  // copies); the handle's stream waits for it
  int rc = PKG_OK;
  {
    HostStager& hs = HostStager::current();
    std::lock_guard<std::mutex> slk(hs.mutex());
    rc = hs.ensure();
    if (!rc) rc = hs.h2d(reinterpret_cast<uint8_t*>(p->witness), witness, 32 * p->nw);
    if (!rc) rc = hs.handoff(p->stream);
  }
  pkg_spartan_proof sp;
  if (!rc)
    rc = pkg_prove_r1cs(&p->r1cs, p->witness, blinding_seed, p->cfg.transcript_domain, &p->whir,
                        &sp, commit_at, proof_at, reinterpret_cast<pkg_stream_t>(p->stream));
  if (rc) {
    free(buf);
    return rc;
  }
  Writer w{buf};
  w.bytes(kProofMagic, 8);
  w.u32(kFormatVersion);
  w.u32(0);
  w.u64(p->m);
  w.u64(p->m0);
  w.u64(p->npub);
  w.u64(nstm);
  w.u64(cwords);
  w.u64(pwords);
  w.u64(p->cfg.transcript_domain);
  w.bytes(&p->whir, 104);
  w.bytes(sp.root, 32);
  w.bytes(sp.r, 32 * p->m0);
  w.bytes(sp.coeffs, 32 * 4 * p->m0);
  w.bytes(sp.alpha, 32 * p->m0);
  w.bytes(sp.rho, 32);
  w.bytes(sp.sum_g, 32);
  w.bytes(sp.blinding_eval, 32);
  w.bytes(sp.public_x, 32);
  w.bytes(sp.evals, 96);
  w.bytes(sp.public_hash, 32);
  w.bytes(sp.public_eval, 32);
  w.bytes(sp.transcript.l, 32);
  w.bytes(sp.transcript.r, 32);
  if (reinterpret_cast<uint8_t*>(commit_at) != w.at) {
    free(buf);
    set_last_error("proof layout mismatch");
    return PKG_ERR_UNSUPPORTED;
  }
  *out_proof = pkg_buf{buf, bytes, bytes};
  return PKG_OK;
}

extern "C" int pkg_prover_serialize(const pkg_prover* p, pkg_buf* out) {
  PK_REQUIRE(out, "null output");
  *out = pkg_buf{nullptr, 0, 0};
  clear_last_error();
  PK_REQUIRE(p, "null prover");
  size_t bytes = 64 + 40;
  for (int k = 0; k < 3; k++)
    bytes += 8 * (p->nc + 1) + align_up(4 * p->nnz[k], 8) + 32 * p->nnz[k];
  uint8_t* buf = static_cast<uint8_t*>(malloc(bytes));
  if (!buf) {
    set_last_error("out of host memory for %zu bytes", bytes);
    return PKG_ERR_OUT_OF_MEMORY;
  }
  Writer w{buf};
  w.bytes(kProverMagic, 8);
  w.u32(kFormatVersion);
  w.u32(0);
  w.u64(p->nc);
  w.u64(p->nw);
  w.u64(p->npub);
  w.u64(p->nnz[0]);
  w.u64(p->nnz[1]);
  w.u64(p->nnz[2]);
  w.u32(p->cfg.folding_factor);
  w.u32(p->cfg.log_inv_rate);
  w.u32(p->cfg.security_bits);
  w.u32(p->cfg.pow_bits);
  w.u32((uint32_t)p->cfg.zk);
  w.u32(0);
  w.u64(p->cfg.transcript_domain);
  w.zeros(8);
  DeviceScope ds(p->device);
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 3 && e == cudaSuccess; k++) {
    e = cudaMemcpy(w.at, p->r1cs.row_ptr[k], 8 * (p->nc + 1), cudaMemcpyDeviceToHost);
    w.at += 8 * (p->nc + 1);
    if (e == cudaSuccess && p->nnz[k])
      e = cudaMemcpy(w.at, p->r1cs.cols[k], 4 * p->nnz[k], cudaMemcpyDeviceToHost);
    w.at += 4 * p->nnz[k];
    w.zeros(align_up(4 * p->nnz[k], 8) - 4 * p->nnz[k]);
    if (e == cudaSuccess && p->nnz[k])
      e = cudaMemcpy(w.at, p->r1cs.vals[k], 32 * p->nnz[k], cudaMemcpyDeviceToHost);
    w.at += 32 * p->nnz[k];
  }
  if (e != cudaSuccess) {
    free(buf);
    return cuda_status(e, "pkg_prover_serialize");
  }
  *out = pkg_buf{buf, bytes, bytes};
  return PKG_OK;
}

extern "C" int pkg_prover_load_bytes(const uint8_t* ptr, size_t len, pkg_prover** out) {
  PK_REQUIRE(out, "null output");
  *out = nullptr;
  clear_last_error();
  PK_REQUIRE(ptr && len, "empty input");
  Reader r{ptr, ptr + len};
  char magic[8];
  uint32_t version = 0, pad = 0;
  uint64_t nc = 0, nw = 0, npub = 0, nnz[3] = {0, 0, 0};
  pkg_prover_config cfg;
  memset(&cfg, 0, sizeof cfg);
  uint32_t c32[6];
  PK_REQUIRE(r.take(magic, 8) && memcmp(magic, kProverMagic, 8) == 0,
             "not a serialized prover (bad magic)");
  PK_REQUIRE(r.take(&version, 4) && version == kFormatVersion, "unsupported prover version %u",
             version);
  PK_REQUIRE(r.take(&pad, 4) && r.take(&nc, 8) && r.take(&nw, 8) && r.take(&npub, 8) &&
                 r.take(nnz, 24) && r.take(c32, 24) && r.take(&cfg.transcript_domain, 8) &&
                 r.skip(8),
             "truncated prover header");
  cfg.folding_factor = c32[0];
  cfg.log_inv_rate = c32[1];
  cfg.security_bits = c32[2];
  cfg.pow_bits = c32[3];
  cfg.zk = (int)c32[4];
  PK_REQUIRE(nc >= 1 && nw >= 1 && nc < (uint64_t(1) << 32) && nw < (uint64_t(1) << 32),
             "bad R1CS dimensions");
  // every array must lie inside the input: sizes checked before any use
  std::vector<uint64_t> rp[3];
  std::vector<uint32_t> cl[3];
  std::vector<uint64_t> vl[3];
  for (int k = 0; k < 3; k++) {
    PK_REQUIRE(nnz[k] < (uint64_t(1) << 40), "matrix %d: implausible nnz %llu", k,
               (unsigned long long)nnz[k]);
    const size_t need = 8 * (nc + 1) + align_up(4 * nnz[k], 8) + 32 * nnz[k];
    PK_REQUIRE((size_t)(r.end - r.at) >= need, "truncated matrix %d", k);
    rp[k].resize(nc + 1);
    cl[k].resize(nnz[k] ? nnz[k] : 1);
    vl[k].resize(4 * (nnz[k] ? nnz[k] : 1));
    r.take(rp[k].data(), 8 * (nc + 1));
    r.take(cl[k].data(), 4 * nnz[k]);
    r.skip(align_up(4 * nnz[k], 8) - 4 * nnz[k]);
    r.take(vl[k].data(), 32 * nnz[k]);
  }
  PK_REQUIRE(r.at == r.end, "%zu trailing bytes after the prover", (size_t)(r.end - r.at));
  const uint64_t* rps[3] = {rp[0].data(), rp[1].data(), rp[2].data()};
  const uint32_t* cls[3] = {cl[0].data(), cl[1].data(), cl[2].data()};
  const uint64_t* vls[3] = {vl[0].data(), vl[1].data(), vl[2].data()};
  const size_t nz[3] = {nnz[0], nnz[1], nnz[2]};
  return pkg_prover_create(nc, nw, npub, rps, cls, vls, nz, &cfg, out);
}
