// rs.cu -- RSFr, provekit's whir ReedSolomon<Fr> plugin
// (provekit/common/src/ntt.rs:12-105), on the device.
//
// interleaved_encode = (1) transpose the messages into the interleaved
// [row][message] layout, (2) append the masks, (3) pick the coset size, (4)
// replicate the first coset num_cosets times, (5) ntt_nr with the first
// log2(num_cosets) stages skipped.  Steps 1, 2 and 4 are one gather kernel
// that writes every codeword slot exactly once; step 5 is the NTT pass
// pipeline of ntt.cu.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "fr.cuh"
#include "fr_host.hpp"
#include "ntt_internal.cuh"
#include "host_stage.cuh"
#include "pk_common.cuh"
#include "rs_internal.cuh"

namespace pk {

// out[o], o in [0, codeword_length*M): x = o mod (coset_size*M);
// x < L*M -> messages[x % M][x / M]; then masks; else 0.
__global__ void rs_gather_kernel(const uint64_t* __restrict__ messages, size_t M, size_t L,
                                 const uint64_t* __restrict__ masks, size_t mask_len,
                                 size_t chunk, size_t total, uint64_t* __restrict__ out) {
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x) {
    size_t x = o % chunk;
    Fr v;
    if (x < L * M) {
      size_t row = x / M, col = x - row * M;
      v = fr_load_ro(messages, col * L + row);
    } else if (x - L * M < mask_len) {
      v = fr_load_ro(masks, x - L * M);
    } else {
      v = fr_zero();
    }
    fr_store(out, o, v);
  }
}

static size_t next_pow2(size_t v) {
  size_t r = 1;
  while (r < v) r <<= 1;
  return r;
}

int rs_plan(size_t num_messages, size_t message_length, size_t mask_len, size_t codeword_length,
            size_t* coset_size_out, size_t* num_cosets_out) {
  size_t total = num_messages * codeword_length;
  PK_REQUIRE(message_length <= codeword_length,
             "message_length %zu exceeds codeword_length %zu", message_length, codeword_length);
  PK_REQUIRE(message_length * num_messages + mask_len <= total,
             "messages + masks (%zu) exceed the codeword (%zu)",
             message_length * num_messages + mask_len, total);
  size_t mask_length = mask_len / num_messages;  // provekit/common/src/ntt.rs:82
  size_t coset_size = next_pow2(message_length + mask_length);
  PK_REQUIRE(coset_size <= (size_t(1) << 28), "coset size exceeds 2^28");
  while (codeword_length % coset_size) {  // ntt.rs:86-89
    coset_size = next_pow2(coset_size + 1);
    PK_REQUIRE(coset_size <= (size_t(1) << 28), "no coset size <= 2^28 divides %zu",
               codeword_length);
  }
  size_t num_cosets = codeword_length / coset_size;
  if (codeword_length > 1) {
    PK_REQUIRE(is_pow2(codeword_length), "codeword_length %zu is not a power of two",
               codeword_length);
  }
  *coset_size_out = coset_size;
  *num_cosets_out = num_cosets;
  return PKG_OK;
}

int rs_encode_device(const uint64_t* messages, size_t num_messages, size_t message_length,
                     const uint64_t* masks, size_t mask_len, size_t codeword_length,
                     uint64_t* out, cudaStream_t stream) {
  if (num_messages == 0) return PKG_OK;  // ntt.rs:57-59
  size_t coset_size = 0, num_cosets = 0;
  int rc = rs_plan(num_messages, message_length, mask_len, codeword_length, &coset_size,
                   &num_cosets);
  if (rc) return rc;
  size_t total = num_messages * codeword_length;
  if (total == 0) return PKG_OK;
  PK_REQUIRE(out != nullptr, "null output pointer");
  PK_REQUIRE(message_length == 0 || messages != nullptr, "null messages pointer");
  PK_REQUIRE(mask_len == 0 || masks != nullptr, "null masks pointer");
  PK_REQUIRE(aligned16(out) && aligned16(messages) && aligned16(masks),
             "device buffers must be 16-byte aligned");
  if (codeword_length > 1 && num_cosets < codeword_length) {
    // the transpose and coset replication are the first NTT pass's loads
    NttSource src;
    src.messages = messages;
    src.masks = masks;
    src.M = num_messages;
    src.L = message_length;
    src.mask_len = mask_len;
    src.chunk = coset_size * num_messages;
    return ntt_nr_from_source(out, total, codeword_length, num_cosets, src, stream);
  }
  int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)sm_count() * 32);
  rs_gather_kernel<<<blocks, 256, 0, stream>>>(messages, num_messages, message_length, masks,
                                               mask_len, coset_size * num_messages, total, out);
  PK_CHECK_LAUNCH("rs_gather_kernel");
  return PKG_OK;
}

// Powers of the order-2^bits root g, split at lo = bits / 2: lo[j] = g^j
// (j < 2^lo) and hi[j] = g^(j 2^lo) (j < 2^(bits - lo)), so g^k is one
// product.  Built once per order on first use (2^lo + 2^(bits - lo)
// products) and kept: every proof opens the same few codeword lengths.
struct PowerTables {
  int lo_bits = 0;
  std::vector<HostFr> lo, hi;
};

static const PowerTables& power_tables(int bits) {
  static std::mutex mu;
  static PowerTables tables[29];
  static bool built[29] = {};
  std::lock_guard<std::mutex> lock(mu);
  PowerTables& t = tables[bits];
  if (!built[bits]) {
    const HostFr g = HostFr::root_of_unity(uint64_t(1) << bits);
    t.lo_bits = bits / 2;
    t.lo.resize(size_t(1) << t.lo_bits);
    t.hi.resize(size_t(1) << (bits - t.lo_bits));
    t.lo[0] = HostFr::one();
    for (size_t j = 1; j < t.lo.size(); j++) t.lo[j] = HostFr::mul(t.lo[j - 1], g);
    const HostFr step = HostFr::mul(t.lo.back(), g);  // g^(2^lo)
    t.hi[0] = HostFr::one();
    for (size_t j = 1; j < t.hi.size(); j++) t.hi[j] = HostFr::mul(t.hi[j - 1], step);
    built[bits] = true;
  }
  return t;
}

}  // namespace pk

using namespace pk;

extern "C" int pkg_rs_next_order(size_t size, size_t* order_out) {
  PK_REQUIRE(order_out != nullptr, "null output");
  size_t order = next_pow2(size);
  if (order > (size_t(1) << 28)) {
    set_last_error("next_order(%zu) exceeds 2^28", size);
    return PKG_ERR_UNSUPPORTED;
  }
  *order_out = order;
  return PKG_OK;
}

extern "C" int pkg_rs_generator(size_t codeword_length, uint64_t out[4]) {
  PK_REQUIRE(out != nullptr, "null output");
  PK_REQUIRE(is_pow2(codeword_length) && codeword_length <= (size_t(1) << 28),
             "no root of unity of order %zu", codeword_length);
  HostFr g = HostFr::root_of_unity(codeword_length);
  memcpy(out, g.l, 32);
  return PKG_OK;
}

extern "C" int pkg_rs_evaluation_points(size_t codeword_length, const size_t* indices, size_t n,
                                        uint64_t* out) {
  PK_REQUIRE(n == 0 || (indices && out), "null pointer");
  PK_REQUIRE(codeword_length >= 1, "codeword_length must be >= 1");
  PK_REQUIRE(is_pow2(codeword_length) && codeword_length <= (size_t(1) << 28),
             "no root of unity of order %zu", codeword_length);
  const int bits = log2_exact(codeword_length);
  const PowerTables& t = power_tables(bits);
  const size_t lo_mask = (size_t(1) << t.lo_bits) - 1;
  for (size_t x = 0; x < n; x++) {
    const size_t i = indices[x];
    size_t k = 0;  // bits = 0: g = 1, every power is 1
    if (bits) {    // i.reverse_bits() >> (usize::BITS - bits)
      size_t r = 0;
      for (int b = 0; b < 64; b++) r |= ((i >> b) & 1) << (63 - b);
      k = r >> (64 - bits);
    }
    const HostFr v = HostFr::mul(t.lo[k & lo_mask], t.hi[k >> t.lo_bits]);
    memcpy(out + 4 * x, v.l, 32);
  }
  return PKG_OK;
}

extern "C" int pkg_rs_interleaved_encode(const uint64_t* messages, size_t num_messages,
                                         size_t message_length, const uint64_t* masks,
                                         size_t mask_len, size_t codeword_length, uint64_t* out,
                                         pkg_stream_t stream) {
  return rs_encode_device(messages, num_messages, message_length, masks, mask_len,
                          codeword_length, out, as_stream(stream));
}

extern "C" int pkg_host_rs_interleaved_encode(const uint64_t* const* messages,
                                              size_t num_messages, size_t message_length,
                                              const uint64_t* masks, size_t mask_len,
                                              size_t codeword_length, uint64_t* out) {
  if (num_messages == 0) return PKG_OK;
  size_t coset_size = 0, num_cosets = 0;
  int rc = rs_plan(num_messages, message_length, mask_len, codeword_length, &coset_size,
                   &num_cosets);
  if (rc) return rc;
  size_t total = num_messages * codeword_length;
  if (total == 0) return PKG_OK;
  PK_REQUIRE(messages != nullptr && out != nullptr, "null pointer");
  PK_REQUIRE(mask_len == 0 || masks != nullptr, "null masks pointer");
  const size_t msg_bytes = 32 * num_messages * message_length, mask_bytes = 32 * mask_len;
  const size_t msg_span = (msg_bytes + 255) & ~size_t(255);
  const size_t mask_span = (mask_bytes + 255) & ~size_t(255);
  HostStager& hs = HostStager::current();
  std::lock_guard<std::mutex> lk(hs.mutex());
  uint8_t* ws = nullptr;
  rc = hs.workspace(msg_span + mask_span + 32 * total, &ws);
  if (rc) return rc;
  uint64_t* d_msg = reinterpret_cast<uint64_t*>(ws);
  uint64_t* d_mask = reinterpret_cast<uint64_t*>(ws + msg_span);
  uint64_t* d_out = reinterpret_cast<uint64_t*>(ws + msg_span + mask_span);
  if (msg_bytes) {
    std::vector<HostSegment> segs(num_messages);
    for (size_t j = 0; j < num_messages; j++) {
      PK_REQUIRE(messages[j] != nullptr, "null message pointer %zu", j);
      segs[j] = HostSegment{messages[j], 32 * message_length};
    }
    rc = hs.h2d(ws, segs.data(), segs.size());
    if (rc) return rc;
  }
  if (mask_bytes) {
    rc = hs.h2d(ws + msg_span, masks, mask_bytes);
    if (rc) return rc;
  }
  rc = rs_encode_device(d_msg, num_messages, message_length, mask_len ? d_mask : nullptr,
                        mask_len, codeword_length, d_out, hs.stream());
  if (rc) return rc;
  rc = hs.d2h(out, reinterpret_cast<uint8_t*>(d_out), 32 * total);
  if (rc) return rc;
  PK_CUDA(cudaStreamSynchronize(hs.stream()));
  return PKG_OK;
}
