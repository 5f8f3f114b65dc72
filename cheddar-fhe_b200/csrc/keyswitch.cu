// Fused key-switching row kernel for N = 2^16.
//
// Between the two fused column passes of a key switch (modswitch.cu) every
// remaining step is row-local in the 128 x 512 limb layout:
//   * the ModUp NTT row phase of every digit (src/core/NTT.cu NTTForModUp),
//   * the key inner product sum_i ModUp(d)_i (.) key_i (Context.cpp:609-647),
//   * the P * (d0, d1) term (Context.cpp:687-699) with the tensor product
//     d0 = b1 b2, d1 = b1 a2 + a1 b2 recomputed from the inputs
//     (ElementWise.cu:504-575), and the own-digit ModUp value d2 = a1 a2,
//   * and, for the primes that ModDown drops, the INTT row phase
//     (NTT.cu:973-1128, INTTForModDown).
// One CTA owns 4 rows of one prime of the extended basis Q u P for one
// ciphertext (each ciphertext names the row tables of its own level, so
// ciphertexts at different levels share a launch); it reads each input row
// once and writes either the
// evaluation-domain accumulator (kept primes, consumed by the ModDown
// epilogue) or the INTT row-phase output (dropped primes, consumed by the
// ModDown column pass).
#include <map>
#include <mutex>
#include <tuple>

#include "arith.cuh"
#include "kernels.h"
#include "ntt_common.cuh"

namespace chd {
namespace {

// PREFETCH: each digit's key words are loaded before its row NTT and the
// next digit's ModUp row during it (more loads in flight per warp, sized for
// 2 CTAs per SM); otherwise each load is issued where it is used, at MINB
// CTAs per SM (3: 80 registers; 4: 64 registers, a few words spilled).  All
// compute the same words; the launcher picks per launch shape.
template <bool PREFETCH, int MINB>
__global__ void __launch_bounds__(256, MINB) k_ks_rows(const __grid_constant__ KSRowsDesc d) {
  __shared__ uint32_t sm[4][512];
  // grid (count, 32, max_rows): the ciphertexts sharing one key row are
  // neighbours in launch order, so the key row comes from HBM once
  const int j = blockIdx.z;
  const KSRowsCt &c = d.ct[blockIdx.x];
  const KSRowsLevel &L = d.lv[c.lv];
  if (j >= L.rows) return;  // a ciphertext below the launch's largest level
  const int g = L.gidx[j];
  const uint32_t q = __ldg(d.primes + g);
  const int32_t qi = __ldg(d.qinvs + g);
  const uint2 *tw = d.tw + (static_cast<size_t>(g) << 16);
  const int t = threadIdx.x & 63, rl = threadIdx.x >> 6;
  const int r = blockIdx.y * 4 + rl;
  uint32_t *srow = sm[rl];
  const size_t off = static_cast<size_t>(j) * 65536 + r * 512 + 8 * t;       // accumulator-row offset
  const size_t koff = static_cast<size_t>(L.key_row[j]) * 65536 + r * 512 + 8 * t;
  const size_t qoff = off;  // input rows share the accumulator row index for q primes
  const bool is_q = j < L.nq;
  const int mode = d.mode;
  uint32_t a1[8], a2[8];
  if (is_q) {
    ld8(c.a1 + qoff, a1);
    if (mode != 1) ld8(c.a2 + qoff, a2);
  }
  uint32_t sb[8], sa[8];
#pragma unroll
  for (int k = 0; k < 8; k++) sb[k] = sa[k] = 0;
  const int own = L.own_digit[j];
  auto load_mu = [&](int i, uint32_t (&x)[8]) {
    const uint32_t *src = c.mu[i] + static_cast<size_t>(j) * 65536 + r * 512;
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = src[t + 64 * k];
  };
  uint32_t vn[8];
  if (PREFETCH && L.beta > 0 && own != 0) load_mu(0, vn);
  for (int i = 0; i < L.beta; i++) {
    uint32_t kb[8], ka[8];
    if (PREFETCH) {
      ld8(L.kb[i] + koff, kb);
      ld8(L.ka[i] + koff, ka);
    }
    uint32_t v[8];
    const bool mine = own == i;
    if (PREFETCH) {
      if (!mine) {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = vn[k];
      }
      if (i + 1 < L.beta && own != i + 1) load_mu(i + 1, vn);
    } else if (!mine) {
      load_mu(i, v);
    }
    if (mine) {
      // own primes of the digit: the ModUp value is the key-switched input
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = mode == 0 ? mont_mul(a1[k], a2[k], q, qi) : (mode == 1 ? a1[k] : a2[k]);
    } else {
      row_fwd(v, srow, tw, r, t, q, 1 + rl);
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = reduce2q(v[k], q);
      row_sync(1 + rl);
    }
    if (!PREFETCH) {
      ld8(L.kb[i] + koff, kb);
      ld8(L.ka[i] + koff, ka);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      sb[k] = add_mod(sb[k], mont_mul(v[k], kb[k], q, qi), q);
      sa[k] = add_mod(sa[k], mont_mul(v[k], ka[k], q, qi), q);
    }
  }
  if (is_q && c.b1 != nullptr) {
    // P * (d0, d1): HMult d0 = b1 b2, d1 = b1 a2 + a1 b2; MultKey d0 = bx;
    // Relinearize d0 = bx, d1 = ax.  Without b1: the bare inner product.
    const uint32_t pp = L.p_prod[j];
    uint32_t b1[8];
    ld8(c.b1 + qoff, b1);
    if (mode == 0) {
      uint32_t b2[8];
      ld8(c.b2 + qoff, b2);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t d0 = mont_mul(b1[k], b2[k], q, qi);
        const uint32_t d1 = mont_mac2(b1[k], a2[k], a1[k], b2[k], q, 0u - static_cast<uint32_t>(qi));
        sb[k] = add_mod(sb[k], mont_mul(d0, pp, q, qi), q);
        sa[k] = add_mod(sa[k], mont_mul(d1, pp, q, qi), q);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        sb[k] = add_mod(sb[k], mont_mul(b1[k], pp, q, qi), q);
        if (mode == 2) sa[k] = add_mod(sa[k], mont_mul(a1[k], pp, q, qi), q);
      }
    }
  }
  const int di = L.drop_idx[j];
  if (di < 0) {
    st8(c.acc_b + off, sb);
    st8(c.acc_a + off, sa);
    return;
  }
  // dropped prime: INTT row phase of both accumulators (ModDown's first step)
  const uint2 *itw = d.itw + (static_cast<size_t>(g) << 16);
  uint32_t *outs[2] = {c.drop_b + static_cast<size_t>(di) * 65536 + r * 512,
                       c.drop_a + static_cast<size_t>(di) * 65536 + r * 512};
#pragma unroll
  for (int p = 0; p < 2; p++) {
    uint32_t *x = p == 0 ? sb : sa;
    row_inv(x, srow, itw, r, t, q, 1 + rl);
#pragma unroll
    for (int k = 0; k < 8; k++) outs[p][t + 64 * k] = x[k];
    row_sync(1 + rl);
  }
}

}  // namespace

namespace {
// Autotuning of the row pass (with the column passes' CHD_BCONV_AUTO): the
// first launch of a shape (device, ciphertexts, largest row count, mode)
// outside a stream capture times the variants three times, interleaved,
// after a warm-up, and caches the fastest; every launch writes the same
// words, so the timing launches leave the right outputs.  Variants: 0 loads
// where used at 3 CTAs per SM, 1 prefetching at 2, 2 loads where used at 4.
constexpr int kKsRowsVariants = 3;
std::mutex g_ksr_mu;
std::map<std::tuple<int, int, int, int>, int> g_ksr_cache;

void launch_variant(const KSRowsDesc &d, int variant, cudaStream_t s) {
  const dim3 grid(d.count, 32, d.max_rows);
  if (variant == 1)
    k_ks_rows<true, 2><<<grid, 256, 0, s>>>(d);
  else if (variant == 2)
    k_ks_rows<false, 4><<<grid, 256, 0, s>>>(d);
  else
    k_ks_rows<false, 3><<<grid, 256, 0, s>>>(d);
}
}  // namespace

void launch_ks_rows(const KSRowsDesc &d, int log_n, cudaStream_t s, bool tune) {
  if (d.count <= 0 || d.max_rows <= 0 || log_n != 16) return;
  if (!tune) {
    launch_variant(d, 0, s);
    return;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, d.count, d.max_rows, d.mode);
  {
    std::lock_guard<std::mutex> lock(g_ksr_mu);
    auto it = g_ksr_cache.find(key);
    if (it != g_ksr_cache.end()) {
      launch_variant(d, it->second, s);
      return;
    }
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    launch_variant(d, 0, s);
    return;
  }
  constexpr int kReps = 3;
  cudaEvent_t ev[kReps * kKsRowsVariants + 1] = {};
  for (auto &e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      for (auto &f : ev)
        if (f) cudaEventDestroy(f);
      launch_variant(d, 0, s);
      return;
    }
  for (int v = 0; v < kKsRowsVariants; v++) launch_variant(d, v, s);
  cudaEventRecord(ev[0], s);
  for (int r = 0; r < kReps; r++)
    for (int v = 0; v < kKsRowsVariants; v++) {
      launch_variant(d, v, s);
      cudaEventRecord(ev[r * kKsRowsVariants + v + 1], s);
    }
  bool ok = cudaEventSynchronize(ev[kReps * kKsRowsVariants]) == cudaSuccess;
  float best[kKsRowsVariants];
  for (float &b : best) b = 1e30f;
  for (int r = 0; ok && r < kReps; r++)
    for (int v = 0; ok && v < kKsRowsVariants; v++) {
      float t = 0.f;
      const int i = r * kKsRowsVariants + v;
      ok = cudaEventElapsedTime(&t, ev[i], ev[i + 1]) == cudaSuccess;
      best[v] = t < best[v] ? t : best[v];
    }
  for (auto &e : ev) cudaEventDestroy(e);
  if (ok) {
    int pick = 0;
    for (int v = 1; v < kKsRowsVariants; v++)
      if (best[v] < best[pick]) pick = v;
    std::lock_guard<std::mutex> lock(g_ksr_mu);
    g_ksr_cache[key] = pick;
  }
}

int ks_rows_tuned_shapes(int *out, int cap) {
  std::lock_guard<std::mutex> lock(g_ksr_mu);
  int k = 0;
  for (const auto &e : g_ksr_cache) {
    if (out && k < cap) {
      out[5 * k] = std::get<0>(e.first);
      out[5 * k + 1] = std::get<1>(e.first);
      out[5 * k + 2] = std::get<2>(e.first);
      out[5 * k + 3] = std::get<3>(e.first);
      out[5 * k + 4] = e.second;
    }
    k++;
  }
  return k;
}

}  // namespace chd
