// Test-only client on the device: secrets, evaluation keys, encryption and
// decryption (the reference's UserInterface, src/UserInterface.cu:110-541,
// which its unit tests use and which it declares not secure).  The
// structure of every key and ciphertext is the reference's; the randomness
// is a seeded counter-based generator, so that key sets of several GB are
// generated in parallel on the GPU and reproduced exactly from the seed.
//
// Randomness: value i of stream S is mix64(S + (i + 1) * gamma), mix64 the
// SplitMix64 finaliser and gamma its golden-ratio increment (G. Steele,
// D. Lea, C. Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014); a stream is mix64(seed ^ mix64(domain)), the domain naming
// the key (kind, rotation) or the encryption nonce and the part (uniform a,
// error e).  Uniform residues are the 64-bit draw mod q (bias below 2^-32);
// errors follow the reference's distribution, round(N(0, 3.2^2)) clamped at
// 6 sigma (include/Random.h:62-75), drawn by inverting its cumulative
// distribution with 64-bit thresholds (integer compares, the same on the
// host and the device).
#include <cmath>
#include <cstring>

#include "../../include/cheddar_b200.h"
#include "arith.cuh"
#include "host.h"
#include "kernels.h"

namespace chd {
namespace {

constexpr uint64_t kGamma = 0x9e3779b97f4a7c15ull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t draw(uint64_t stream, uint64_t i) { return mix64(stream + (i + 1) * kGamma); }
uint64_t stream_of(uint64_t seed, uint64_t domain) { return mix64(seed ^ mix64(domain)); }

// domains: kind in the top byte, then the rotation / nonce, then the part
uint64_t domain(int kind, uint64_t idx, int part) {
  return (static_cast<uint64_t>(kind) << 56) ^ (idx << 8) ^ static_cast<uint64_t>(part);
}
enum Kind { kSecretDense = 1, kSecretSparse, kMult, kConj, kRot, kDts, kStd, kEncrypt };

// error distribution: P(e <= k) for k = -19 .. 19 as 64-bit thresholds
constexpr int kErrMax = 19;  // llround of the 6-sigma clamp 19.2
struct ErrTable {
  uint64_t t[2 * kErrMax + 1];  // t[k + 19] = floor(P(e <= k) 2^64), last = all ones
};
ErrTable make_err_table() {
  const double sd = 3.2, clamp = 6 * sd;
  ErrTable et{};
  // P(e <= k) = P(X < k + 0.5) (round half away from zero, X continuous);
  // the clamp sends |X| > 19.2 to +-19
  auto cdf = [&](double x) { return 0.5 * std::erfc(-x / (sd * std::sqrt(2.0))); };
  for (int k = -kErrMax; k <= kErrMax; k++) {
    double p = k == kErrMax ? 1.0 : cdf(std::fmin(k + 0.5, clamp));
    if (k == -kErrMax) p = cdf(-kErrMax + 0.5);
    et.t[k + kErrMax] = p >= 1.0 ? ~uint64_t{0} : static_cast<uint64_t>(std::ldexp(p, 64));
  }
  return et;
}
__host__ __device__ __forceinline__ int sample_err(uint64_t u, const ErrTable &et) {
  int k = 0;
  while (k < 2 * kErrMax && u >= et.t[k]) k++;
  return k - kErrMax;
}

struct ClientRows {
  uint32_t q[64];
  int32_t qinv[64];
  int gidx[64];       // global prime of each row (the secret's row)
  uint32_t pprod[64];  // Montgomery P mod q on the rows a digit adds its target to
  int rows, n;
};

// out[r][j] = uniform residue of row r
__global__ void k_uniform(uint32_t *out, const __grid_constant__ ClientRows cr, uint64_t stream, uint64_t base) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const uint64_t idx = base + (static_cast<uint64_t>(cr.gidx[r]) * cr.n + j);
  out[static_cast<size_t>(r) * cr.n + j] = static_cast<uint32_t>(draw(stream, idx) % cr.q[r]);
}
// out[r][j] = the same small error coefficient j on every row (coefficient domain)
__global__ void k_error(uint32_t *out, const __grid_constant__ ClientRows cr, uint64_t stream, uint64_t base,
                        const __grid_constant__ ErrTable et) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const int e = sample_err(draw(stream, base + j), et);
  const uint32_t q = cr.q[r];
  out[static_cast<size_t>(r) * cr.n + j] = e < 0 ? q - static_cast<uint32_t>(-e) : static_cast<uint32_t>(e);
}
// bx = e - a s_enc (+ target P on rows [t0, t1)), UserInterface.cu:57-108
__global__ void k_evk_part(uint32_t *bx, const uint32_t *ax, const uint32_t *e, const uint32_t *s_enc,
                           const uint32_t *target, const __grid_constant__ ClientRows cr, int t0, int t1) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const size_t k = static_cast<size_t>(r) * cr.n + j, ks = static_cast<size_t>(cr.gidx[r]) * cr.n + j;
  const uint32_t q = cr.q[r];
  uint32_t v = sub_mod(e[k], mont_mul(ax[k], s_enc[ks], q, cr.qinv[r]), q);
  if (r >= t0 && r < t1) v = add_mod(v, mont_mul(target[ks], cr.pprod[r], q, cr.qinv[r]), q);
  bx[k] = v;
}
// bx = m - a s + e (Encrypt, UserInterface.cu:17-55)
__global__ void k_encrypt(uint32_t *bx, const uint32_t *ax, const uint32_t *m, const uint32_t *e, const uint32_t *s,
                          const __grid_constant__ ClientRows cr) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const size_t k = static_cast<size_t>(r) * cr.n + j, ks = static_cast<size_t>(cr.gidx[r]) * cr.n + j;
  const uint32_t q = cr.q[r];
  bx[k] = add_mod(sub_mod(m[k], mont_mul(ax[k], s[ks], q, cr.qinv[r]), q), e[k], q);
}
// m = b + a s (Decrypt, UserInterface.cu:185-206)
__global__ void k_decrypt(uint32_t *m, const uint32_t *bx, const uint32_t *ax, const uint32_t *s,
                          const __grid_constant__ ClientRows cr) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const size_t k = static_cast<size_t>(r) * cr.n + j, ks = static_cast<size_t>(cr.gidx[r]) * cr.n + j;
  const uint32_t q = cr.q[r];
  m[k] = add_mod(bx[k], mont_mul(ax[k], s[ks], q, cr.qinv[r]), q);
}
// x = a (.) b (Montgomery), over every row of the full basis
__global__ void k_mont_square(uint32_t *out, const uint32_t *a, const __grid_constant__ ClientRows cr) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const size_t k = static_cast<size_t>(r) * cr.n + j;
  out[k] = mont_mul(a[k], a[k], cr.q[r], cr.qinv[r]);
}
// dst_0 += dst_i over digits (ElementWiseHandler::Accum of the
// sparse-to-dense key's digits, UserInterface.cu:345-352)
__global__ void k_accum_digits(uint32_t *x, size_t words, int beta, const __grid_constant__ ClientRows cr) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (j >= cr.n) return;
  const size_t k = static_cast<size_t>(r) * cr.n + j;
  uint32_t v = x[k];
  for (int i = 1; i < beta; i++) v = add_mod(v, x[i * words + k], cr.q[r]);
  x[k] = v;
}

dim3 grid_of(const ClientRows &cr) { return dim3((cr.n + 255) / 256, cr.rows); }

}  // namespace

// ---- the client ----------------------------------------------------------------

struct Client {
  Context *ctx = nullptr;
  uint64_t seed = 0;
  NP full;                         // max-level key basis: all q primes + alpha aux
  uint32_t *dense = nullptr;       // [full.total][N], NTT Montgomery
  uint32_t *sparse = nullptr;      // same, with sparse-secret encapsulation
  ErrTable et{};
  ~Client() {
    cudaFree(dense);
    cudaFree(sparse);
  }
};

namespace {

ClientRows rows_of(const Context &C, const NP &np) {
  ClientRows cr{};
  cr.rows = np.total();
  cr.n = C.P->n;
  C.P->gidx(np, cr.gidx);
  for (int r = 0; r < cr.rows; r++) {
    cr.q[r] = C.P->primes[cr.gidx[r]];
    cr.qinv[r] = C.P->qinv[cr.gidx[r]];
  }
  return cr;
}

// UserInterface::PrepareSecrets (UserInterface.cu:224-276): h distinct
// positions (partial Fisher-Yates), values +-1, residues on every prime of
// the key basis, NTT with the Montgomery conversion
Status make_secret(Context &C, uint64_t seed, int kind, int h, uint32_t **out) {
  const int n = C.P->n;
  CHD_CHECK(h >= 1 && h <= n, kErrInvalidArg, "client: Hamming weight out of range");
  const uint64_t sp = stream_of(seed, domain(kind, 0, 0)), ss = stream_of(seed, domain(kind, 0, 1));
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  for (int i = 0; i < h; i++) {
    const int j = i + static_cast<int>(draw(sp, i) % static_cast<uint64_t>(n - i));
    std::swap(idx[i], idx[j]);
  }
  const NP full = C.P->level_np(C.P->max_level, C.P->alpha);
  const int tot = full.total();
  std::vector<int> g(tot);
  C.P->gidx(full, g.data());
  std::vector<uint32_t> s(static_cast<size_t>(tot) * n, 0);
  for (int r = 0; r < tot; r++) {
    const uint32_t p = C.P->primes[g[r]];
    for (int i = 0; i < h; i++) s[static_cast<size_t>(r) * n + idx[i]] = (draw(ss, i) & 1) ? p - 1 : 1u;
  }
  CHD_CHECK(cudaMalloc(out, s.size() * 4) == cudaSuccess, kErrAlloc, "client: secret allocation failed");
  cudaMemcpyAsync(*out, s.data(), s.size() * 4, cudaMemcpyHostToDevice, C.stream);
  CHD_TRY(C.ntt(full, *out, true));
  return cudaStreamSynchronize(C.stream) == cudaSuccess ? kOk : kErrCuda;
}

// UserInterface::PrepareEvk (UserInterface.cu:366-458) over key basis np:
// enc and target are full-basis secrets (rows by global prime)
Status make_evk(Context &C, Client &cl, int kind, uint64_t idx, const NP &np, const uint32_t *enc,
                const uint32_t *target, DeviceEvk *k) {
  const int n = C.P->n, nq = np.q(), tot = np.total();
  CHD_CHECK(np.aux >= 1 && tot <= 64, kErrInvalidArg, "client: invalid key basis");
  const int beta = (nq + np.aux - 1) / np.aux;
  CHD_CHECK(beta <= 8, kErrUnsupported, "client: more than 8 digits");
  ClientRows cr = rows_of(C, np);
  // P = product of the basis' aux primes, on the q rows (Montgomery)
  for (int r = 0; r < nq; r++) {
    uint32_t v = 1;
    for (int a = 0; a < np.aux; a++) v = prime::mul_mod(v, C.P->primes[cr.gidx[nq + a]], cr.q[r]);
    cr.pprod[r] = prime::to_mont(v, cr.q[r]);
  }
  const size_t words = static_cast<size_t>(tot) * n;
  k->beta = beta;
  k->np = np;
  CHD_CHECK(cudaMalloc(&k->bx, beta * words * 4) == cudaSuccess && cudaMalloc(&k->ax, beta * words * 4) == cudaSuccess,
            kErrAlloc, "client: key allocation failed");
  ArenaScope scope(C.arena);
  uint32_t *e = static_cast<uint32_t *>(C.arena.alloc(words * 4));
  CHD_CHECK(e, kErrAlloc, "client: scratch allocation failed");
  const uint64_t sa = stream_of(cl.seed, domain(kind, idx, 2)), se = stream_of(cl.seed, domain(kind, idx, 3));
  for (int i = 0; i < beta; i++) {
    uint32_t *ax = k->ax + i * words, *bx = k->bx + i * words;
    k_uniform<<<grid_of(cr), 256, 0, C.stream>>>(ax, cr, sa, static_cast<uint64_t>(i) * 64 * n);
    k_error<<<grid_of(cr), 256, 0, C.stream>>>(e, cr, se, static_cast<uint64_t>(i) * n, cl.et);
    CHD_TRY(C.ntt(np, e, true));
    const int t0 = i * np.aux, t1 = std::min((i + 1) * np.aux, nq);
    k_evk_part<<<grid_of(cr), 256, 0, C.stream>>>(bx, ax, e, enc, target, cr, t0, t1);
  }
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_error(std::string("client key: ") + cudaGetErrorString(err));
    return kErrCuda;
  }
  return kOk;
}

// a full-basis secret permuted by the automorphism of `amount` (N/2 - r for
// a rotation by r, -1 for conjugation), ElementWiseHandler::Permute
Status permuted_secret(Context &C, const uint32_t *s, int amount, uint32_t *out) {
  const NP full = C.P->level_np(C.P->max_level, C.P->alpha);
  const int tot = full.total(), n = C.P->n;
  std::vector<int> g(tot);
  C.P->gidx(full, g.data());
  PermuteBatch pb{};
  pb.galois = C.P->galois_of(amount);
  for (int r = 0; r < tot; r++) {
    if (pb.count == kMaxPermuteRows) {
      launch_permute(pb, C.P->log_n, C.stream);
      pb.count = 0;
    }
    PermuteRow &pr = pb.rows[pb.count++];
    pr.src = s + static_cast<size_t>(r) * n;
    pr.dst = out + static_cast<size_t>(r) * n;
    pr.add = nullptr;
    pr.src2 = nullptr;
    pr.q = C.P->primes[g[r]];
  }
  launch_permute(pb, C.P->log_n, C.stream);
  return kOk;
}

}  // namespace
}  // namespace chd

// ---- C ABI ----------------------------------------------------------------------

struct chd_client {
  chd::Client c;
};

namespace {
using namespace chd;

int client_fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

#define CLIENT_GUARD(ctx, cl)                                                              \
  if (!(ctx) || !(cl)) return client_fail(CHD_ERR_INVALID_ARG, "client: null argument"); \
  DeviceGuard device_guard_((ctx)->c->device)

// Builds a key over np with the given secrets and hands it to the C ABI.
int finish_key(chd_context *ctx, chd_client *cl, int kind, uint64_t idx, const NP &np, const uint32_t *enc,
               const uint32_t *target, chd_evk **out, bool accumulate_digits) {
  Context &C = *ctx->c;
  DeviceEvk k;
  int rc = make_evk(C, cl->c, kind, idx, np, enc, target, &k);
  if (rc != kOk) return rc;
  if (accumulate_digits && k.beta > 1) {
    ClientRows cr = rows_of(C, np);
    const size_t words = static_cast<size_t>(np.total()) * C.P->n;
    k_accum_digits<<<grid_of(cr), 256, 0, C.stream>>>(k.bx, words, k.beta, cr);
    k_accum_digits<<<grid_of(cr), 256, 0, C.stream>>>(k.ax, words, k.beta, cr);
  }
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return client_fail(CHD_ERR_CUDA, "client: key generation failed");
  rc = chd_evk_create_np(ctx, np.main, np.ter, np.aux, accumulate_digits ? 1 : k.beta, k.bx, k.ax, 1, out);
  return rc;
}

}  // namespace

extern "C" {

int chd_client_create(chd_context *ctx, uint64_t seed, chd_client **out) try {
  if (!ctx || !out) return client_fail(CHD_ERR_INVALID_ARG, "chd_client_create: null argument");
  Context &C = *ctx->c;
  DeviceGuard device_guard(C.device);
  auto *cl = new chd_client();
  cl->c.ctx = &C;
  cl->c.seed = seed;
  cl->c.full = C.P->level_np(C.P->max_level, C.P->alpha);
  cl->c.et = make_err_table();
  int rc = make_secret(C, seed, kSecretDense, C.dense_hw(), &cl->c.dense);
  if (rc == kOk && C.uses_sse()) rc = make_secret(C, seed, kSecretSparse, C.P->spec.sparse_hw, &cl->c.sparse);
  if (rc != kOk) {
    delete cl;
    return rc;
  }
  *out = cl;
  return CHD_OK;
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_create: ") + e.what());
}

void chd_client_destroy(chd_client *cl) { delete cl; }

int chd_client_secret(chd_context *ctx, const chd_client *cl, int sparse, uint32_t *out) try {
  CLIENT_GUARD(ctx, cl);
  const uint32_t *s = sparse ? cl->c.sparse : cl->c.dense;
  if (!out || !s) return client_fail(CHD_ERR_INVALID_ARG, "chd_client_secret: no such secret");
  const size_t words = static_cast<size_t>(cl->c.full.total()) * ctx->c->P->n;
  if (cudaMemcpy(out, s, words * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return client_fail(CHD_ERR_CUDA, "chd_client_secret: copy failed");
  return CHD_OK;
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_secret: ") + e.what());
}

int chd_client_mult_key(chd_context *ctx, chd_client *cl, chd_evk **out) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  const size_t words = static_cast<size_t>(cl->c.full.total()) * C.P->n;
  ArenaScope scope(C.arena);
  uint32_t *s2 = static_cast<uint32_t *>(C.arena.alloc(words * 4));
  if (!s2) return client_fail(CHD_ERR_ALLOC, "chd_client_mult_key: scratch allocation failed");
  ClientRows cr = rows_of(C, cl->c.full);
  k_mont_square<<<grid_of(cr), 256, 0, C.stream>>>(s2, cl->c.dense, cr);
  return finish_key(ctx, cl, kMult, 0, cl->c.full, cl->c.dense, s2, out, false);
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_mult_key: ") + e.what());
}

int chd_client_rotation_key(chd_context *ctx, chd_client *cl, int rot_idx, chd_evk **out) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  if (rot_idx <= 0 || rot_idx >= C.P->n / 2)
    return client_fail(CHD_ERR_INVALID_ARG, "chd_client_rotation_key: rotation index must be in [1, N/2)");
  const size_t words = static_cast<size_t>(cl->c.full.total()) * C.P->n;
  ArenaScope scope(C.arena);
  uint32_t *sr = static_cast<uint32_t *>(C.arena.alloc(words * 4));
  if (!sr) return client_fail(CHD_ERR_ALLOC, "chd_client_rotation_key: scratch allocation failed");
  permuted_secret(C, cl->c.dense, C.P->n / 2 - rot_idx, sr);
  return finish_key(ctx, cl, kRot, static_cast<uint64_t>(rot_idx), cl->c.full, sr, cl->c.dense, out, false);
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_rotation_key: ") + e.what());
}

int chd_client_conjugation_key(chd_context *ctx, chd_client *cl, chd_evk **out) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  const size_t words = static_cast<size_t>(cl->c.full.total()) * C.P->n;
  ArenaScope scope(C.arena);
  uint32_t *sc = static_cast<uint32_t *>(C.arena.alloc(words * 4));
  if (!sc) return client_fail(CHD_ERR_ALLOC, "chd_client_conjugation_key: scratch allocation failed");
  permuted_secret(C, cl->c.dense, -1, sc);
  return finish_key(ctx, cl, kConj, 0, cl->c.full, sc, cl->c.dense, out, false);
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_conjugation_key: ") + e.what());
}

int chd_client_sse_keys(chd_context *ctx, chd_client *cl, chd_evk **dense_to_sparse, chd_evk **sparse_to_dense) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  if (!cl->c.sparse) return client_fail(CHD_ERR_UNSUPPORTED, "chd_client_sse_keys: parameters without encapsulation");
  // dense-to-sparse over the level -1 primes and as many aux primes
  // (UserInterface.cu:523-529), sparse-to-dense over the full basis with its
  // digits summed into one (UserInterface.cu:335-352)
  NP dts = C.P->level_np(-1);
  dts.aux = dts.q();
  int rc = finish_key(ctx, cl, kDts, 0, dts, cl->c.sparse, cl->c.dense, dense_to_sparse, false);
  if (rc != CHD_OK) return rc;
  return finish_key(ctx, cl, kStd, 0, cl->c.full, cl->c.dense, cl->c.sparse, sparse_to_dense, true);
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_sse_keys: ") + e.what());
}

int chd_client_encrypt(chd_context *ctx, chd_client *cl, uint64_t nonce, int level, double scale, int num_slots,
                       const uint32_t *pt_dev, chd_ciphertext *ct) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  if (!pt_dev || !ct) return client_fail(CHD_ERR_INVALID_ARG, "chd_client_encrypt: null argument");
  if (level < -1 || level > C.P->max_level) return client_fail(CHD_ERR_INVALID_LEVEL, "chd_client_encrypt: invalid level");
  const NP np = C.P->level_np(level);
  int rc = chd_ct_import(ctx, ct, np.main, np.ter, 0, 0, scale, num_slots, pt_dev, pt_dev, nullptr, 1);
  if (rc != CHD_OK) return rc;
  uint32_t *bx = nullptr, *ax = nullptr, *rx = nullptr;
  chd_ct_device_ptrs(ct, &bx, &ax, &rx);
  ClientRows cr = rows_of(C, np);
  const size_t words = static_cast<size_t>(np.total()) * C.P->n;
  ArenaScope scope(C.arena);
  uint32_t *e = static_cast<uint32_t *>(C.arena.alloc(words * 4));
  if (!e) return client_fail(CHD_ERR_ALLOC, "chd_client_encrypt: scratch allocation failed");
  k_uniform<<<grid_of(cr), 256, 0, C.stream>>>(ax, cr, stream_of(cl->c.seed, domain(kEncrypt, nonce, 2)), 0);
  k_error<<<grid_of(cr), 256, 0, C.stream>>>(e, cr, stream_of(cl->c.seed, domain(kEncrypt, nonce, 3)), 0, cl->c.et);
  rc = C.ntt(np, e, true);
  if (rc != kOk) return rc;
  k_encrypt<<<grid_of(cr), 256, 0, C.stream>>>(bx, ax, pt_dev, e, cl->c.dense, cr);
  return cudaStreamSynchronize(C.stream) == cudaSuccess ? CHD_OK
                                                        : client_fail(CHD_ERR_CUDA, "chd_client_encrypt: failed");
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_encrypt: ") + e.what());
}

int chd_client_decrypt(chd_context *ctx, const chd_client *cl, const chd_ciphertext *ct, uint32_t *pt_dev) try {
  CLIENT_GUARD(ctx, cl);
  Context &C = *ctx->c;
  if (!pt_dev || !ct) return client_fail(CHD_ERR_INVALID_ARG, "chd_client_decrypt: null argument");
  int m = 0, t = 0, a = 0, has_rx = 0, ns = 0;
  double sc = 0;
  chd_ct_info(ct, &m, &t, &a, &has_rx, &sc, &ns);
  if (a != 0 || has_rx) return client_fail(CHD_ERR_SHAPE, "chd_client_decrypt: relinearised ciphertext without aux primes required");
  uint32_t *bx = nullptr, *ax = nullptr, *rx = nullptr;
  chd_ct_device_ptrs(ct, &bx, &ax, &rx);
  ClientRows cr = rows_of(C, NP{m, t, 0});
  k_decrypt<<<grid_of(cr), 256, 0, C.stream>>>(pt_dev, bx, ax, cl->c.dense, cr);
  return cudaStreamSynchronize(C.stream) == cudaSuccess ? CHD_OK
                                                        : client_fail(CHD_ERR_CUDA, "chd_client_decrypt: failed");
} catch (const std::exception &e) {
  return client_fail(CHD_ERR_INTERNAL, std::string("chd_client_decrypt: ") + e.what());
}

}  // extern "C"
