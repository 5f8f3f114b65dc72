// Fused ModSwitch column pass with the base conversion on the tcgen05
// tensor cores (INT8 limbs, exact), N = 2^16.
//
// Same dataflow as k_modswitch_cols (modswitch.cu): per 16-column tile the
// K sources go through the INTT column stages, the output constant and
// centring; every target is base-converted, taken through the NTT column
// stages and written once.  The base conversion
//   V[m][n] = sum_k x_k[n] T[m][k]   (x centred, T the centred table)
// runs as byte-limb MMAs instead of 64-bit multiply-adds:
//   * the sources are stored offset, x' = x + 2^30 in [0, 2^31), so that
//     their four bytes are plain unsigned digits (A operand, u8);
//   * B holds the bytes of c[m][k][j] = 2^(8j) T[m][k] mod p_m (u8): row
//     4m + i of B is byte i of c, K byte 4k + j pairs with byte j of x'_k;
//   * D[n][4m + i] = sum_(k, j) byte_j(x'_k) byte_i(c[m][k][j]) < 2^22 is
//     exact in int32, and sum_i 2^(8i) D[n][4m + i] + corr_m (< 2^48) with
//     corr_m = -2^30 sum_k T[m][k] mod p_m is congruent to V[m][n].
// One Montgomery reduction then gives the canonical residue of
// V * 2^-32 mod p_m, the value the CUDA-core column pass produces: the two
// passes are bit-identical.
//
// Thread t holds element e (e = 0..15) of its column, so MMA e (M = 128
// coefficients, N = 16 = 4 targets x 4 bytes) takes A row t from thread t's
// e-th source values, and TMEM lane t of accumulator e comes back to the
// same thread: the converted values land in the registers where the NTT
// column stages need them, with no exchange.  Targets go in chunks of four,
// each in two halves of 8 slots (128 TMEM columns per CTA, so that three
// CTAs share an SM); the MMAs of the next chunk's first half run while the
// CUDA cores transform the current chunk.
#include <algorithm>

#include "arith.cuh"
#include "colpass.cuh"
#include "kernels.h"
#include "ntt_common.cuh"
#include "tc_common.cuh"

namespace chd {
namespace {

using namespace tc;

constexpr int32_t kOffset = 1 << 30;  // makes centred sources non-negative
constexpr uint32_t kTmemCols = 128;   // 8 accumulators of 16 columns (half a chunk)

// A operand of one slot e: 32-byte K steps of 128 rows (4096 B, core
// matrices of 8 rows x 16 B, LBO 128, SBO 256).  With KMAX = 12 the last
// step holds 4 sources (16 bytes per row) in 2048 B: SBO 128, and its upper
// 16-byte K half (LBO 128) reads the next row group, finite values that meet
// the zero bytes of B there.
template <int KMAX>
struct Geo {
  static constexpr int kFull = KMAX / 8;
  static constexpr int kHalf = (KMAX % 8) ? 1 : 0;
  static constexpr int kSteps = kFull + kHalf;
  static constexpr int kSlotBytes = kFull * 4096 + kHalf * 2048;
  static constexpr int kBBytes = kSteps * 512;  // one B chunk: 16 rows x 32 B per step
  static constexpr int kSmem = kExRows * kTC * 4 + 16 * kSlotBytes + 2 * kBBytes + 32;
};

// kind::i8: D s32 (bits 4-5 = 2), A u8 and B u8 (bits 7-9, 10-12 = 0), both
// K-major, N = 16 (N >> 3 at bit 17), M = 128 (M >> 4 at bit 24)
constexpr uint32_t kIdesc = (2u << 4) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// Sources KMAX .. KMAX + KR - 1 (K = 13, 14) stay in registers and are
// converted on the CUDA cores in the epilogue (one more Montgomery chunk),
// so that they need neither A bytes nor the next larger KMAX.
template <int KMAX, int KR>
__global__ void __launch_bounds__(128, KMAX <= 8 ? 3 : 2) k_modswitch_cols_tc(const __grid_constant__ MSColBatch b) {
  using G = Geo<KMAX>;
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const MSColJob &jb = b.jobs[blockIdx.y];
  uint32_t *ex = reinterpret_cast<uint32_t *>(smem);
  uint8_t *sa = smem + kExRows * kTC * 4;
  uint8_t *sb = sa + 16 * G::kSlotBytes;
  uint32_t *corr = reinterpret_cast<uint32_t *>(sb + 2 * G::kBBytes);
  const uint32_t sa_u = smem_u32(sa), sb_u = smem_u32(sb), bar = smem_u32(&mbar);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int cl = lane & 15, rg = 2 * w + (lane >> 4);
  const int col = blockIdx.x * kTC + cl;
  const int K = jb.K, M = jb.M;
  const int Kt = K < KMAX ? K : KMAX;  // sources on the tensor cores
  const int nch = (M + 3) >> 2;
  int32_t xr[KR > 0 ? KR : 1][16];     // sources in registers (centred)

  // both B buffers start zero: rows of missing targets and K bytes past the
  // sources stay zero
  for (int i = t; i < G::kBBytes / 2; i += 128) reinterpret_cast<uint32_t *>(sb)[i] = 0;
  if (t == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = static_cast<uint32_t>(32 * w) << 16;

  // B operand and offset correction of target chunk c into buffer buf
  auto build_b = [&](int c, int buf) {
    uint8_t *bb = sb + buf * G::kBBytes;
    if (t < 4 * Kt) {
      const int mq = t / Kt, k = t - mq * Kt;
      const int m = 4 * c + mq;
      uint32_t cj[4] = {0u, 0u, 0u, 0u};
      if (m < M) {
        const uint32_t p = __ldg(b.primes + jb.dst_gidx[m]);
        const int32_t tv = __ldg(jb.table + m * K + k);
        uint32_t x = tv < 0 ? static_cast<uint32_t>(tv + static_cast<int32_t>(p)) : static_cast<uint32_t>(tv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
          cj[j] = x;
#pragma unroll
          for (int s = 0; s < 8; s++) {  // x * 256 mod p by doublings (x < p < 2^31)
            x <<= 1;
            x = x >= p ? x - p : x;
          }
        }
      }
      const int s = k >> 3, bo = 4 * (k & 7);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int n = 4 * mq + i;
        const uint32_t word = ((cj[0] >> (8 * i)) & 0xffu) | (((cj[1] >> (8 * i)) & 0xffu) << 8) |
                              (((cj[2] >> (8 * i)) & 0xffu) << 16) | (((cj[3] >> (8 * i)) & 0xffu) << 24);
        *reinterpret_cast<uint32_t *>(bb + s * 512 + (n >> 3) * 256 + (bo >> 4) * 128 + (n & 7) * 16 + (bo & 15)) =
            word;
      }
    }
    if (t < 4) {
      const int m = 4 * c + t;
      uint32_t cv = 0;
      if (m < M) {
        const uint32_t p = __ldg(b.primes + jb.dst_gidx[m]);
        uint32_t sum = 0;
        for (int k = 0; k < Kt; k++) {
          const int32_t tv = __ldg(jb.table + m * K + k);
          sum = add_mod(sum, tv < 0 ? static_cast<uint32_t>(tv + static_cast<int32_t>(p)) : static_cast<uint32_t>(tv),
                        p);
        }
        for (int s = 0; s < 30; s++) {  // 2^30 * sum mod p
          sum <<= 1;
          sum = sum >= p ? sum - p : sum;
        }
        cv = sum ? p - sum : 0u;
      }
      corr[buf * 4 + t] = cv;
    }
  };

  // one thread: the MMAs of half a chunk (slots 8 half .. 8 half + 7) into
  // the 8 accumulators, then commit
  auto issue = [&](int buf, int half) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
    for (int e = 8 * half; e < 8 * half + 8; e++) {
#pragma unroll
      for (int s = 0; s < G::kSteps; s++) {
        const uint32_t aaddr = sa_u + e * G::kSlotBytes + s * 4096;
        const uint64_t ad = smem_desc(aaddr, 128, s < G::kFull ? 256 : 128);
        const uint64_t bd = smem_desc(sb_u + buf * G::kBBytes + s * 512, 128, 256);
        const uint32_t acc = s > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem + 16u * (e & 7)),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
  };

  // ---- phase A: INTT column stages, output constant, centring, offset; the
  // A rows are written four sources (16 bytes) at a time
  for (int kg = 0; kg < K; kg += 4) {
    uint32_t xw[4][16];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int k = kg + kk;
      if (k < K) {
        const int g = jb.src_gidx[k];
        const uint32_t q = __ldg(b.primes + g);
        const uint2 *itw = b.itw + (static_cast<size_t>(g) << 16);
        const uint32_t *src = jb.src + (static_cast<size_t>(jb.src_row[k]) << 16);
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
          const int j = 2 * rg + hh;
          uint32_t y[8];
#pragma unroll
          for (int u = 0; u < 8; u++) y[u] = __ldg(src + (8 * j + u) * 512 + col);
          radix8_inv(y, itw, 16 + j, 32 + 2 * j, 64 + 4 * j, q);
#pragma unroll
          for (int u = 0; u < 8; u++) ex[exi(8 * j + u, cl)] = y[u];
        }
        __syncthreads();
        uint32_t x[16];
#pragma unroll
        for (int e = 0; e < 16; e++) x[e] = ex[exi(rg + 8 * e, cl)];
        radix16_cols_inv(x, itw, q);
        const uint32_t c0 = jb.c0[k], c0s = jb.c0s[k];
#pragma unroll
        for (int e = 0; e < 16; e++) {
          const int32_t xc = centre(reduce2q(shoup_lazy(x[e], c0, c0s, q), q), q);
          xw[kk][e] = static_cast<uint32_t>(xc + kOffset);
#pragma unroll
          for (int r = 0; r < KR; r++)
            if (k == KMAX + r) xr[r][e] = xc;
        }
        __syncthreads();
      } else {
#pragma unroll
        for (int e = 0; e < 16; e++) xw[kk][e] = 0u;
      }
    }
    if (kg >= KMAX) continue;  // register sources
    const int s = kg >> 3, bo = 4 * (kg & 7);
    const int roff = s < G::kFull ? s * 4096 + (t >> 3) * 256 + (bo >> 4) * 128 + (t & 7) * 16 : s * 4096 + t * 16;
#pragma unroll
    for (int e = 0; e < 16; e++)
      *reinterpret_cast<uint4 *>(sa + e * G::kSlotBytes + roff) = make_uint4(xw[0][e], xw[1][e], xw[2][e], xw[3][e]);
  }
  build_b(0, 0);
  // make the generic-proxy stores visible to the tensor core
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (t == 0) issue(0, 0);

  // ---- phase B: per chunk of 4 targets, TMEM -> residues -> NTT column
  // stages -> HBM (radix-16 stages of two targets interleaved)
  auto finish = [&](int m, const uint32_t (&v)[16]) {
    const int g = jb.dst_gidx[m];
    const uint32_t p = __ldg(b.primes + g);
    const uint2 *tw = b.tw + (static_cast<size_t>(g) << 16);
#pragma unroll
    for (int e = 0; e < 16; e++) ex[exi(rg + 8 * e, cl)] = v[e];
    __syncthreads();
    uint32_t *dst = jb.dst + (static_cast<size_t>(jb.dst_row[m]) << 16);
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const int j = 2 * rg + hh;
      uint32_t y[8];
#pragma unroll
      for (int u = 0; u < 8; u++) y[u] = ex[exi(8 * j + u, cl)];
      radix8_fwd(y, tw, 16 + j, 32 + 2 * j, 64 + 4 * j, p);
#pragma unroll
      for (int u = 0; u < 8; u++) dst[(8 * j + u) * 512 + col] = y[u];
    }
    __syncthreads();
  };
  uint32_t phase = 0;
  bool ok = true;
  for (int c = 0; c < nch && ok; c++) {
    const int buf = c & 1;
    uint32_t p[4];
    int32_t pinv[4];
    uint32_t v[4][16];
#pragma unroll
    for (int half = 0; half < 2; half++) {
      // every thread polls with a limit; the CTA leaves together if any gave up
      if (!__syncthreads_and(mbar_wait(bar, phase) ? 1 : 0)) {
        ok = false;
        break;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // the MMAs that read buffer buf ^ 1 (chunk c - 1) have completed
      if (half == 0 && c + 1 < nch) build_b(c + 1, buf ^ 1);
      uint32_t cr[4];
      int32_t tr[4][KR > 0 ? KR : 1];
#pragma unroll
      for (int mq = 0; mq < 4; mq++) {
        const int m = 4 * c + mq;
        const int g = m < M ? jb.dst_gidx[m] : 0;
        p[mq] = m < M ? __ldg(b.primes + g) : 1u;
        pinv[mq] = m < M ? __ldg(b.qinvs + g) : 1;
        cr[mq] = corr[buf * 4 + mq];
#pragma unroll
        for (int r = 0; r < KR; r++) tr[mq][r] = m < M && KMAX + r < K ? __ldg(jb.table + m * K + KMAX + r) : 0;
      }
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        uint32_t r[32];
        tmem_ld32(tmem + lane_base + 16u * e, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int mq = 0; mq < 4; mq++) {
            const uint32_t *d = r + 16 * h + 4 * mq;
            const uint32_t lo = d[0] + (d[1] << 8) + cr[mq];
            const uint32_t hi = d[2] + (d[3] << 8);
            const uint64_t val = (static_cast<uint64_t>(hi) << 16) + lo;
            uint32_t res = mont_reduce(static_cast<int64_t>(val), p[mq], pinv[mq]);
            if (KR > 0) {
              int64_t a = 0;
#pragma unroll
              for (int r = 0; r < KR; r++) a += static_cast<int64_t>(xr[r][8 * half + e + h]) * tr[mq][r];
              res = add_mod(res, mont_reduce(a, p[mq], pinv[mq]), p[mq]);
            }
            v[mq][8 * half + e + h] = res;
          }
      }
      // accumulators read (and B of chunk c + 1 written): the next MMAs may start
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (t == 0) {
        if (half == 0)
          issue(buf, 1);
        else if (c + 1 < nch)
          issue(buf ^ 1, 0);
      }
    }
    if (!ok) break;
#pragma unroll
    for (int mq = 0; mq < 4; mq += 2) {
      const int m = 4 * c + mq;
      if (m + 1 < M) {
        const uint2 *tw0 = b.tw + (static_cast<size_t>(jb.dst_gidx[m]) << 16);
        const uint2 *tw1 = b.tw + (static_cast<size_t>(jb.dst_gidx[m + 1]) << 16);
        radix16_cols_fwd(v[mq], tw0, p[mq]);  // stages m = 1, 2, 4, 8 on rows rg + 8e
        radix16_cols_fwd(v[mq + 1], tw1, p[mq + 1]);
        finish(m, v[mq]);
        finish(m + 1, v[mq + 1]);
      } else if (m < M) {
        radix16_cols_fwd(v[mq], b.tw + (static_cast<size_t>(jb.dst_gidx[m]) << 16), p[mq]);
        finish(m, v[mq]);
      }
    }
  }
  if (!ok) {
    if (t == 0 && b.err) atomicExch(b.err, 1);
    // a second bounded chance for the MMAs in flight before TMEM is freed
    mbar_wait(bar, phase);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (w == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

template <int KMAX, int KR>
void launch_kmax(const MSColBatch &b, cudaStream_t s) {
  // CTAs per SM: 3 for KMAX = 8 (shared memory and registers), 2 for 12, 1
  // for 16; their accumulators (128 TMEM columns each) always fit
  const size_t sm = Geo<KMAX>::kSmem;
  cudaFuncSetAttribute(k_modswitch_cols_tc<KMAX, KR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(sm));
  k_modswitch_cols_tc<KMAX, KR><<<dim3(512 / kTC, b.count), 128, sm, s>>>(b);
}

}  // namespace

size_t modswitch_cols_tc_smem(int kmax) {
  return kmax <= 8 ? Geo<8>::kSmem : (kmax <= 12 ? Geo<12>::kSmem : Geo<16>::kSmem);
}

void launch_modswitch_cols_tc(const MSColBatch &b, int max_k, cudaStream_t s) {
  if (b.count <= 0) return;
  if (max_k <= 8)
    launch_kmax<8, 0>(b, s);
  else if (max_k <= 12)
    launch_kmax<12, 0>(b, s);
  else if (max_k <= 14)
    launch_kmax<12, 2>(b, s);
  else
    launch_kmax<16, 0>(b, s);
}

}  // namespace chd
