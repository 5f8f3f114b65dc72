// Residue serialization: a stable byte format for ciphertexts and evaluation
// keys (the reference has none; its objects live only in device memory).
//
// Little-endian, 8-byte aligned sections:
//   ciphertext:  "CHDCT001" | u32 log_n, num_main, num_ter, num_aux, has_rx,
//                num_slots | f64 scale | u32 rows, u32 pad | u32 prime[rows]
//                (padded to 8 bytes) | parts bx, ax[, rx], each [rows][N] u32
//   key:         "CHDEVK01" | u32 log_n, beta, num_main, num_ter, num_aux, rows
//                | u32 prime[rows] (padded) | bx [beta][rows][N] | ax [beta][rows][N]
// The residues are the in-memory layout of this library and of the
// reference (prime order terminal reversed, main, aux; canonical, NTT
// Montgomery domain), so a buffer is the ciphertext or key itself plus the
// primes it is defined over; loading checks them against the context.
#include <cstring>

#include "../../include/cheddar_b200.h"
#include "host.h"

namespace chd {
namespace {

constexpr char kCtMagic[8] = {'C', 'H', 'D', 'C', 'T', '0', '0', '1'};
constexpr char kEvkMagic[8] = {'C', 'H', 'D', 'E', 'V', 'K', '0', '1'};

size_t pad8(size_t x) { return (x + 7) & ~size_t{7}; }

struct Writer {
  uint8_t *p;
  size_t cap, len = 0;
  void put(const void *src, size_t n) {
    if (p && len + n <= cap) std::memcpy(p + len, src, n);
    len += n;
  }
  void u32(uint32_t v) { put(&v, 4); }
  void align() {
    static const uint8_t z[8] = {};
    put(z, pad8(len) - len);
  }
};

struct Reader {
  const uint8_t *p;
  size_t len, pos = 0;
  bool get(void *dst, size_t n) {
    if (pos + n > len) return false;
    std::memcpy(dst, p + pos, n);
    pos += n;
    return true;
  }
  bool u32(uint32_t *v) { return get(v, 4); }
  void align() { pos = pad8(pos); }
};

// primes of np's rows, checked against a stored list
bool same_primes(const Params &P, const NP &np, const std::vector<uint32_t> &stored) {
  std::vector<int> g(np.total());
  P.gidx(np, g.data());
  if (stored.size() != g.size()) return false;
  for (size_t i = 0; i < g.size(); i++)
    if (P.primes[g[i]] != stored[i]) return false;
  return true;
}

}  // namespace
}  // namespace chd

using namespace chd;

namespace {
int ser_fail(int code, const std::string &m) {
  set_error(m);
  return code;
}
}  // namespace

extern "C" {

int chd_ct_serialize(chd_context *ctx, const chd_ciphertext *ct, void *buf, size_t cap, size_t *len) try {
  if (!ctx || !ct || !len) return ser_fail(CHD_ERR_INVALID_ARG, "chd_ct_serialize: null argument");
  Context &C = *ctx->c;
  DeviceGuard guard(C.device);
  const DeviceCt &c = ct->ct;
  const int rows = c.np.total(), n = C.P->n;
  Writer w{static_cast<uint8_t *>(buf), buf ? cap : 0};
  w.put(kCtMagic, 8);
  const uint32_t hdr[6] = {static_cast<uint32_t>(C.P->log_n), static_cast<uint32_t>(c.np.main),
                           static_cast<uint32_t>(c.np.ter), static_cast<uint32_t>(c.np.aux),
                           c.has_rx ? 1u : 0u, static_cast<uint32_t>(c.num_slots)};
  w.put(hdr, sizeof hdr);
  w.put(&c.scale, 8);
  w.u32(static_cast<uint32_t>(rows));
  w.u32(0);
  std::vector<int> g(rows);
  C.P->gidx(c.np, g.data());
  for (int r = 0; r < rows; r++) w.u32(C.P->primes[g[r]]);
  w.align();
  const size_t part = static_cast<size_t>(rows) * n * 4;
  const size_t body = w.len;
  const int parts = c.has_rx ? 3 : 2;
  w.len += parts * part;
  *len = w.len;
  if (!buf) return CHD_OK;
  if (cap < w.len) return ser_fail(CHD_ERR_INVALID_ARG, "chd_ct_serialize: buffer too small");
  const uint32_t *src[3] = {c.bx, c.ax, c.rx};
  for (int i = 0; i < parts; i++)
    cudaMemcpyAsync(static_cast<uint8_t *>(buf) + body + i * part, src[i], part, cudaMemcpyDeviceToHost, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : ser_fail(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return ser_fail(CHD_ERR_INTERNAL, std::string("chd_ct_serialize: ") + e.what());
}

int chd_ct_deserialize(chd_context *ctx, chd_ciphertext *ct, const void *buf, size_t len) try {
  if (!ctx || !ct || !buf) return ser_fail(CHD_ERR_INVALID_ARG, "chd_ct_deserialize: null argument");
  Context &C = *ctx->c;
  DeviceGuard guard(C.device);
  Reader r{static_cast<const uint8_t *>(buf), len};
  char magic[8];
  uint32_t hdr[6], rows = 0, pad = 0;
  double scale = 0;
  if (!r.get(magic, 8) || std::memcmp(magic, kCtMagic, 8) != 0)
    return ser_fail(CHD_ERR_PARSE, "chd_ct_deserialize: not a ciphertext buffer");
  if (!r.get(hdr, sizeof hdr) || !r.get(&scale, 8) || !r.u32(&rows) || !r.u32(&pad))
    return ser_fail(CHD_ERR_PARSE, "chd_ct_deserialize: truncated header");
  if (hdr[0] != static_cast<uint32_t>(C.P->log_n))
    return ser_fail(CHD_ERR_SHAPE, "chd_ct_deserialize: ring degree differs from the context's");
  const NP np{static_cast<int>(hdr[1]), static_cast<int>(hdr[2]), static_cast<int>(hdr[3])};
  if (np.main > C.P->max_main || np.ter > C.P->max_ter || np.aux > C.P->alpha || rows != static_cast<uint32_t>(np.total()))
    return ser_fail(CHD_ERR_SHAPE, "chd_ct_deserialize: prime counts outside the context");
  std::vector<uint32_t> primes(rows);
  for (auto &p : primes)
    if (!r.u32(&p)) return ser_fail(CHD_ERR_PARSE, "chd_ct_deserialize: truncated prime list");
  if (!same_primes(*C.P, np, primes)) return ser_fail(CHD_ERR_SHAPE, "chd_ct_deserialize: primes differ from the context's");
  r.align();
  const int n = C.P->n, parts = hdr[4] ? 3 : 2;
  const size_t part = static_cast<size_t>(rows) * n * 4;
  if (r.pos + parts * part != len) return ser_fail(CHD_ERR_PARSE, "chd_ct_deserialize: residue section has the wrong size");
  const uint8_t *body = static_cast<const uint8_t *>(buf) + r.pos;
  return chd_ct_import(ctx, ct, np.main, np.ter, np.aux, hdr[4] ? 1 : 0, scale, static_cast<int>(hdr[5]),
                       reinterpret_cast<const uint32_t *>(body), reinterpret_cast<const uint32_t *>(body + part),
                       hdr[4] ? reinterpret_cast<const uint32_t *>(body + 2 * part) : nullptr, 0);
} catch (const std::exception &e) {
  return ser_fail(CHD_ERR_INTERNAL, std::string("chd_ct_deserialize: ") + e.what());
}

int chd_evk_serialize(chd_context *ctx, const chd_evk *evk, void *buf, size_t cap, size_t *len) try {
  if (!ctx || !evk || !len) return ser_fail(CHD_ERR_INVALID_ARG, "chd_evk_serialize: null argument");
  Context &C = *ctx->c;
  DeviceGuard guard(C.device);
  const DeviceEvk &k = evk->k;
  const int rows = k.np.total(), n = C.P->n;
  Writer w{static_cast<uint8_t *>(buf), buf ? cap : 0};
  w.put(kEvkMagic, 8);
  const uint32_t hdr[6] = {static_cast<uint32_t>(C.P->log_n), static_cast<uint32_t>(k.beta),
                           static_cast<uint32_t>(k.np.main), static_cast<uint32_t>(k.np.ter),
                           static_cast<uint32_t>(k.np.aux), static_cast<uint32_t>(rows)};
  w.put(hdr, sizeof hdr);
  std::vector<int> g(rows);
  C.P->gidx(k.np, g.data());
  for (int r = 0; r < rows; r++) w.u32(C.P->primes[g[r]]);
  w.align();
  const size_t part = static_cast<size_t>(k.beta) * rows * n * 4;
  const size_t body = w.len;
  w.len += 2 * part;
  *len = w.len;
  if (!buf) return CHD_OK;
  if (cap < w.len) return ser_fail(CHD_ERR_INVALID_ARG, "chd_evk_serialize: buffer too small");
  cudaMemcpyAsync(static_cast<uint8_t *>(buf) + body, k.bx, part, cudaMemcpyDeviceToHost, C.stream);
  cudaMemcpyAsync(static_cast<uint8_t *>(buf) + body + part, k.ax, part, cudaMemcpyDeviceToHost, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : ser_fail(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return ser_fail(CHD_ERR_INTERNAL, std::string("chd_evk_serialize: ") + e.what());
}

int chd_evk_deserialize(chd_context *ctx, const void *buf, size_t len, chd_evk **out) try {
  if (!ctx || !buf || !out) return ser_fail(CHD_ERR_INVALID_ARG, "chd_evk_deserialize: null argument");
  Context &C = *ctx->c;
  DeviceGuard guard(C.device);
  Reader r{static_cast<const uint8_t *>(buf), len};
  char magic[8];
  uint32_t hdr[6];
  if (!r.get(magic, 8) || std::memcmp(magic, kEvkMagic, 8) != 0)
    return ser_fail(CHD_ERR_PARSE, "chd_evk_deserialize: not a key buffer");
  if (!r.get(hdr, sizeof hdr)) return ser_fail(CHD_ERR_PARSE, "chd_evk_deserialize: truncated header");
  if (hdr[0] != static_cast<uint32_t>(C.P->log_n))
    return ser_fail(CHD_ERR_SHAPE, "chd_evk_deserialize: ring degree differs from the context's");
  const NP np{static_cast<int>(hdr[2]), static_cast<int>(hdr[3]), static_cast<int>(hdr[4])};
  const uint32_t rows = hdr[5];
  if (rows != static_cast<uint32_t>(np.total()) || np.main > C.P->max_main || np.ter > C.P->max_ter)
    return ser_fail(CHD_ERR_SHAPE, "chd_evk_deserialize: prime counts outside the context");
  std::vector<uint32_t> primes(rows);
  for (auto &p : primes)
    if (!r.u32(&p)) return ser_fail(CHD_ERR_PARSE, "chd_evk_deserialize: truncated prime list");
  if (!same_primes(*C.P, np, primes)) return ser_fail(CHD_ERR_SHAPE, "chd_evk_deserialize: primes differ from the context's");
  r.align();
  const size_t part = static_cast<size_t>(hdr[1]) * rows * C.P->n * 4;
  if (r.pos + 2 * part != len) return ser_fail(CHD_ERR_PARSE, "chd_evk_deserialize: residue section has the wrong size");
  const uint8_t *body = static_cast<const uint8_t *>(buf) + r.pos;
  return chd_evk_create_np(ctx, np.main, np.ter, np.aux, static_cast<int>(hdr[1]),
                           reinterpret_cast<const uint32_t *>(body), reinterpret_cast<const uint32_t *>(body + part), 0,
                           out);
} catch (const std::exception &e) {
  return ser_fail(CHD_ERR_INTERNAL, std::string("chd_evk_deserialize: ") + e.what());
}

}  // extern "C"
