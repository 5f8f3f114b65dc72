// ModUp that allocates no device memory.
//
// chd_modup_raw takes its scratch (the centred INTT output of the input
// limbs) from the context's device arena, which grows with cudaMalloc the
// first time a larger operation needs it.  Some callers must not allocate
// device memory once they are running: latency-critical servers (a
// cudaMalloc can synchronise the device and stall every other stream), and
// hosts whose device memory is owned by another allocator or capped by a
// fixed budget.  chd_modup_raw_noalloc serves them: its scratch is the
// file-scope device array below, sized once for the whole process.
//
// Limits and sharing:
//   * capacity kNoAllocScratchWords 32-bit words (8 MiB): num_q(level) * N
//     must not exceed it (32 q primes at N = 2^16); larger requests fail with
//     CHD_ERR_UNSUPPORTED;
//   * every GPU that loads the library holds the array until the process
//     exits;
//   * all calls share the array, so calls whose GPU work overlaps (other
//     streams, other contexts on the same device) race; the scratch is fully
//     written before it is read, so nothing needs clearing between calls;
//   * the array's device address is looked up once per device, on the
//     first call for a context of that device (the call makes the context's
//     device current while it runs); make that first call before any stream
//     capture.
#include <cstdint>
#include <exception>
#include <mutex>

#include "../../include/cheddar_b200.h"
#include "host.h"

namespace chd {
namespace {

constexpr size_t kNoAllocScratchWords = size_t{1} << 21;
static __device__ __align__(256) uint32_t g_modup_scratch[kNoAllocScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t *g_scratch_addr[kMaxDevices] = {};

// Device address of g_modup_scratch on `device`, which must be the current
// device (looked up once per device).
Status scratch_address(int device, uint32_t **out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("chd_modup_raw_noalloc: device index out of range");
    return kErrInvalidArg;
  }
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != device) {
    set_error("chd_modup_raw_noalloc: the context's device is not current");
    return kErrCuda;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_modup_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("chd_modup_raw_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return kErrCuda;
    }
    g_scratch_addr[device] = static_cast<uint32_t *>(p);
  }
  *out = g_scratch_addr[device];
  return kOk;
}

// N < 2^16: INTT (centred, times (N q-hat)^-1) into the scratch, copy of the
// digit's own primes, BConv, NTT — the unfused ModUp of ModSwitch.cu:429-509.
Status modup_small(Context &C, int level, const uint32_t *src, uint32_t *const *dst, uint32_t *xt) {
  const LevelMS &m = C.lms(level);
  const int n = C.P->n;
  NP np = C.P->level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  // k_bconv holds at most 16 sources and 64 targets per job, as in
  // Context::modup_many: check every digit before any work is issued
  for (int i = 0; i < m.beta; i++) {
    const int s = m.dig_s[i], e = m.dig_e[i];
    if (e > 0 && (e - s > 16 || tot - (e - s) > 64)) {
      set_error("chd_modup_raw_noalloc: a digit of more than 16 primes or more than 64 targets");
      return kErrUnsupported;
    }
  }
  int g[256];
  C.P->gidx(np, g);
  RowBatch rb{};
  auto flush = [&](bool fwd) {
    if (!rb.count) return;
    if (fwd)
      launch_ntt_fwd(rb, C.P->log_n, C.stream);
    else
      launch_ntt_inv(rb, C.P->log_n, C.stream);
    rb.count = 0;
  };
  for (int r = 0; r < nq; r++) {
    RowDesc &d = rb.rows[rb.count++];
    d = RowDesc{};
    d.src = src + static_cast<size_t>(r) * n;
    d.dst = xt + static_cast<size_t>(r) * n;
    d.tw = C.itw(g[r]);
    d.q = C.P->primes[g[r]];
    C.mont_as_shoup(m.mod_up1[r], g[r], &d.c0, &d.c0s);
    d.flags = kCentre;
    if (rb.count == kMaxRows) flush(false);
  }
  flush(false);
  BConvBatch b{};
  b.primes = C.d_primes;
  b.qinvs = C.d_qinv;
  for (int i = 0; i < m.beta; i++) {
    const int s = m.dig_s[i], e = m.dig_e[i];
    if (e <= 0) continue;
    cudaMemcpyAsync(dst[i] + static_cast<size_t>(s) * n, src + static_cast<size_t>(s) * n,
                    static_cast<size_t>(e - s) * n * 4, cudaMemcpyDeviceToDevice, C.stream);
    BConvJob &j = b.jobs[b.count++];
    j.xt = reinterpret_cast<const int32_t *>(xt) + static_cast<size_t>(s) * n;
    j.out = dst[i];
    j.table = m.d_mod_up2[i];
    j.K = e - s;
    j.M = tot - (e - s);
    int k = 0;
    for (int r = 0; r < tot; r++) {
      if (r >= s && r < e) continue;
      j.out_row[k] = static_cast<uint8_t>(r);
      j.out_gidx[k] = static_cast<uint8_t>(g[r]);
      k++;
    }
    if (b.count == kMaxBConvJobs) {
      launch_bconv(b, C.P->log_n, C.stream);
      b.count = 0;
    }
  }
  launch_bconv(b, C.P->log_n, C.stream);
  for (int i = 0; i < m.beta; i++) {
    const int s = m.dig_s[i], e = m.dig_e[i];
    if (e <= 0) continue;
    for (int r = 0; r < tot; r++) {
      if (r >= s && r < e) continue;
      RowDesc &d = rb.rows[rb.count++];
      d = RowDesc{};
      d.src = d.dst = dst[i] + static_cast<size_t>(r) * n;
      d.tw = C.tw(g[r]);
      d.q = C.P->primes[g[r]];
      if (rb.count == kMaxRows) flush(true);
    }
  }
  flush(true);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("chd_modup_raw_noalloc: ") + cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

}  // namespace
}  // namespace chd

extern "C" int chd_modup_raw_noalloc(chd_context *ctx, int level, const uint32_t *src_dev,
                                     uint32_t *dst_dev) try {
  using namespace chd;
  if (!ctx || !src_dev || !dst_dev) {
    set_error("chd_modup_raw_noalloc: null argument");
    return CHD_ERR_INVALID_ARG;
  }
  // the kernels move device data in 16-byte vectors
  if ((reinterpret_cast<uintptr_t>(src_dev) | reinterpret_cast<uintptr_t>(dst_dev)) & 15) {
    set_error("chd_modup_raw_noalloc: device pointers must be 16-byte aligned");
    return CHD_ERR_INVALID_ARG;
  }
  Context &C = *ctx->c;
  DeviceGuard device_guard(C.device);
  if (level < -1 || level > C.P->max_level) {
    set_error("chd_modup_raw_noalloc: invalid level");
    return CHD_ERR_INVALID_LEVEL;
  }
  const LevelMS &m = C.lms(level);
  const size_t words = static_cast<size_t>(m.num_q) * C.P->n;
  if (words > kNoAllocScratchWords) {
    set_error("chd_modup_raw_noalloc: num_q * N = " + std::to_string(words) +
              " words exceeds the static scratch of " + std::to_string(kNoAllocScratchWords) + " words");
    return CHD_ERR_UNSUPPORTED;
  }
  if (m.beta > 8) {
    set_error("chd_modup_raw_noalloc: more than 8 digits");
    return CHD_ERR_UNSUPPORTED;
  }
  uint32_t *scratch = nullptr;
  Status st = scratch_address(C.device, &scratch);
  if (st != kOk) return st;
  const size_t stride = static_cast<size_t>(m.num_q + m.num_aux) * C.P->n;
  uint32_t *dst[8];
  for (int i = 0; i < m.beta; i++) dst[i] = dst_dev + i * stride;
  if (C.P->log_n == 16) {
    const uint32_t *srcs[1] = {src_dev};
    uint32_t *const *dsts[1] = {dst};
    return C.modup_fused(level, 1, srcs, dsts, scratch);
  }
  return modup_small(C, level, src_dev, dst, scratch);
} catch (const std::exception &e) {
  chd::set_error(std::string("chd_modup_raw_noalloc: internal error: ") + e.what());
  return CHD_ERR_INTERNAL;
} catch (...) {
  chd::set_error("chd_modup_raw_noalloc: internal error");
  return CHD_ERR_INTERNAL;
}
