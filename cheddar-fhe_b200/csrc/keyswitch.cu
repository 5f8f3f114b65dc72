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
#include "arith.cuh"
#include "kernels.h"
#include "ntt_common.cuh"

namespace chd {
namespace {

// Per-thread staging of one digit's operands, filled by cp.async one digit
// ahead: the thread's 8 ModUp values (elements t + 64k of its row, words
// [k][256 threads]) and its 8 + 8 key words (as 4 x 16 bytes,
// [chunk][256 threads]), so the loads of digit i + 1 fly while digit i's
// row NTT runs.  Two buffers of 24 KiB, then 16 KiB for the thread's b1 and
// b2 words of the P * (d0, d1) term, fetched with the first digit.
constexpr int kStageWords = 8 * 256 + 4 * 256 * 4;
constexpr int kStageBytes = (2 * kStageWords + 4 * 256 * 4) * 4;

__device__ __forceinline__ void cp_async4(uint32_t *dst, const uint32_t *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(256, 3) k_ks_rows(const __grid_constant__ KSRowsDesc d) {
  __shared__ uint32_t sm[4][512];
  extern __shared__ uint4 stage_raw[];
  uint32_t *stage = reinterpret_cast<uint32_t *>(stage_raw);
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
  const int tid = threadIdx.x;
  const int own = L.own_digit[j];
  // issue digit i's copies into buffer i & 1
  auto prefetch = [&](int i) {
    uint32_t *st = stage + (i & 1) * kStageWords;
    if (own != i) {
      const uint32_t *src = c.mu[i] + static_cast<size_t>(j) * 65536 + r * 512;
#pragma unroll
      for (int k = 0; k < 8; k++) cp_async4(st + k * 256 + tid, src + t + 64 * k);
    }
    uint4 *kst = reinterpret_cast<uint4 *>(st + 8 * 256);
    const uint4 *kb = reinterpret_cast<const uint4 *>(L.kb[i] + koff);
    const uint4 *ka = reinterpret_cast<const uint4 *>(L.ka[i] + koff);
    cp_async16(kst + 0 * 256 + tid, kb);
    cp_async16(kst + 1 * 256 + tid, kb + 1);
    cp_async16(kst + 2 * 256 + tid, ka);
    cp_async16(kst + 3 * 256 + tid, ka + 1);
    cp_async_commit();
  };
  uint4 *bst = reinterpret_cast<uint4 *>(stage + 2 * kStageWords);
  const bool with_p = is_q && c.b1 != nullptr;
  if (with_p) {
    const uint4 *b1 = reinterpret_cast<const uint4 *>(c.b1 + qoff);
    cp_async16(bst + tid, b1);
    cp_async16(bst + 256 + tid, b1 + 1);
    if (mode == 0) {
      const uint4 *b2 = reinterpret_cast<const uint4 *>(c.b2 + qoff);
      cp_async16(bst + 512 + tid, b2);
      cp_async16(bst + 768 + tid, b2 + 1);
    }
  }
  if (L.beta > 0)
    prefetch(0);  // its commit closes the group with b1 / b2
  else
    cp_async_commit();
  for (int i = 0; i < L.beta; i++) {
    if (i + 1 < L.beta) {
      prefetch(i + 1);
      cp_async_wait<1>();  // digit i's group has landed (the thread's own words)
    } else {
      cp_async_wait<0>();
    }
    const uint32_t *st = stage + (i & 1) * kStageWords;
    uint32_t v[8];
    if (own == i) {
      // own primes of the digit: the ModUp value is the key-switched input
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = mode == 0 ? mont_mul(a1[k], a2[k], q, qi) : (mode == 1 ? a1[k] : a2[k]);
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = st[k * 256 + tid];
      row_fwd(v, srow, tw, r, t, q, 1 + rl);
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = reduce2q(v[k], q);
      row_sync(1 + rl);
    }
    const uint4 *kst = reinterpret_cast<const uint4 *>(st + 8 * 256);
    const uint4 b0 = kst[tid], b1v = kst[256 + tid], a0 = kst[512 + tid], a1v = kst[768 + tid];
    const uint32_t kb[8] = {b0.x, b0.y, b0.z, b0.w, b1v.x, b1v.y, b1v.z, b1v.w};
    const uint32_t ka[8] = {a0.x, a0.y, a0.z, a0.w, a1v.x, a1v.y, a1v.z, a1v.w};
#pragma unroll
    for (int k = 0; k < 8; k++) {
      sb[k] = add_mod(sb[k], mont_mul(v[k], kb[k], q, qi), q);
      sa[k] = add_mod(sa[k], mont_mul(v[k], ka[k], q, qi), q);
    }
  }
  cp_async_wait<0>();
  if (with_p) {
    // P * (d0, d1): HMult d0 = b1 b2, d1 = b1 a2 + a1 b2; MultKey d0 = bx;
    // Relinearize d0 = bx, d1 = ax.  Without b1: the bare inner product.
    // (The last wait above covered every group, the first one included.)
    const uint32_t pp = L.p_prod[j];
    const uint4 x0 = bst[tid], x1 = bst[256 + tid];
    const uint32_t b1[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
    if (mode == 0) {
      const uint4 y0 = bst[512 + tid], y1 = bst[768 + tid];
      const uint32_t b2[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
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

void launch_ks_rows(const KSRowsDesc &d, int log_n, cudaStream_t s) {
  if (d.count <= 0 || d.max_rows <= 0 || log_n != 16) return;
  constexpr int smem = kStageBytes;  // 64 KiB of staging beside the 8 KiB row buffers
  cudaFuncSetAttribute(k_ks_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k_ks_rows<<<dim3(d.count, 32, d.max_rows), 256, smem, s>>>(d);
}

}  // namespace chd
