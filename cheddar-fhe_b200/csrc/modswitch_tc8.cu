// Fused ModSwitch column pass on the tcgen05 tensor cores with 256-thread
// tiles (8 coefficients per thread), N = 2^16.
//
// The same dataflow and the same words as k_modswitch_cols_tc
// (modswitch_tc.cu): per 16-column tile the K sources go through the INTT
// column stages, the output constant and centring, are stored as unsigned
// bytes (x + 2^30) into the A operand, the base conversion runs as byte-limb
// MMAs into int32 TMEM accumulators, and each target is Montgomery-reduced,
// taken through the NTT column stages and written once.
//
// What differs is the thread layout.  There a thread holds 16 elements of a
// column, and 168-194 registers per thread and the K-source A operand in
// shared memory leave 2-3 warps per scheduler, which the butterflies'
// dependent chains cannot keep busy.  Here a thread holds 8 elements, so a
// tile has twice the threads at half the registers:
//   layout 1 (global loads and stores, the stages at row distances 1, 2, 4):
//     thread (w, lane) holds rows 8 j + u (u = 0..7) of column lane % 16,
//     j = 2 w + lane / 16, as in the 128-thread pass;
//   layout 2 (the stages at row distances 8, 16, 32): rows w + 8 e + 64 h
//     (e = 0..7), h = lane / 16;
//   the stage at row distance 64 (m = 1) pairs lanes l and l ^ 16 of one
//     warp and runs through a shuffle: on the inverse side it is fused with
//     the output constant (c0 for row r, c0 w1 for row r + 64), on the
//     forward side each half multiplies by 1 or w1 before the exchange.
// A layout change goes through an 8 KiB exchange buffer whose XOR swizzle
// keeps both access patterns free of bank conflicts.  Element e of thread
// (w, lane) is A row / TMEM lane 32 (w % 4) + lane of slot 2 e + w / 4, and
// slot s's accumulator sits at TMEM column 64 (s % 2) + 16 ((s / 2) % 4): the
// four slots a thread reads in one half-chunk are adjacent columns of its
// own lane quarter (warp w may only read lanes 32 (w % 4) ...).
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
constexpr int kThreads = 256;

// A operand of one slot: as in modswitch_tc.cu (32-byte K steps of 128
// rows, core matrices of 8 rows x 16 B, LBO 128, SBO 256; a trailing half
// step of 4 sources, SBO 128)
template <int KMAX>
struct Geo8 {
  static constexpr int kFull = KMAX / 8;
  static constexpr int kHalf = (KMAX % 8) ? 1 : 0;
  static constexpr int kSteps = kFull + kHalf;
  static constexpr int kSlotBytes = kFull * 4096 + kHalf * 2048;
  static constexpr int kBBytes = kSteps * 512;  // one B chunk: 16 rows x 32 B per step
  static constexpr int kExBytes = 128 * kTC * 4;
  static constexpr int kSmem = kExBytes + 16 * kSlotBytes + 2 * kBBytes + 64;
};

// kind::i8: D s32, A u8, B u8, both K-major, N = 16, M = 128
constexpr uint32_t kIdesc = (2u << 4) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// exchange-buffer word of (row, column): rows r and r + 8 (layout 1) and r
// and r + 64 (layout 2) land in opposite bank halves
__device__ __forceinline__ int xsw(int row, int c) {
  return (row * kTC + c) ^ ((((row >> 3) ^ (row >> 6)) & 1) << 4);
}

__device__ __forceinline__ uint32_t acc_col(int s) { return 64u * (s & 1) + 16u * ((s >> 1) & 3); }

// MINB: CTAs per SM the register budget is sized for (3: 80 registers, 2:
// 128); KMAX = 8 fits 3 CTAs in shared memory, KMAX = 12 only 2
template <int KMAX, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_modswitch_cols_tc8(const __grid_constant__ MSColBatch b) {
  using G = Geo8<KMAX>;
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ uint2 c0w[16];  // (c0 w1 mod q, Shoup companion) per source
  const MSColJob &jb = b.jobs[blockIdx.y];
  uint32_t *ex = reinterpret_cast<uint32_t *>(smem);
  uint8_t *sa = smem + G::kExBytes;
  uint8_t *sb = sa + 16 * G::kSlotBytes;
  uint32_t *corr = reinterpret_cast<uint32_t *>(sb + 2 * G::kBBytes);  // [2][4]
  uint32_t *ones = corr + 8;                                            // [2][4]: floor(2^32 / p)
  const uint32_t sa_u = smem_u32(sa), sb_u = smem_u32(sb), bar = smem_u32(&mbar);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int cl = lane & 15, hb = lane >> 4;
  const int col = blockIdx.x * kTC + cl;
  const int j1 = 2 * w + hb;          // layout 1: rows 8 j1 + u
  const int R = 32 * (w & 3) + lane;  // A row and TMEM lane of this thread
  const int g2 = w >> 2;              // element e lives in slot 2 e + g2
  const int K = jb.K, M = jb.M;
  const int nch = (M + 3) >> 2;

  for (int i = t; i < G::kBBytes / 2; i += kThreads) reinterpret_cast<uint32_t *>(sb)[i] = 0;
  if (t < K) {
    const int g = jb.src_gidx[t];
    const uint32_t q = __ldg(b.primes + g);
    const uint32_t w1 = __ldg(b.itw + (static_cast<size_t>(g) << 16) + 1).x;
    const uint32_t v = static_cast<uint32_t>(static_cast<uint64_t>(jb.c0[t]) * w1 % q);
    c0w[t] = make_uint2(v, static_cast<uint32_t>((static_cast<uint64_t>(v) << 32) / q));
  }
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
  const uint32_t lane_base = static_cast<uint32_t>(32 * (w & 3)) << 16;

  // B operand, offset correction and floor(2^32 / p) of target chunk c
  auto build_b = [&](int c, int buf) {
    uint8_t *bb = sb + buf * G::kBBytes;
    if (t < 4 * K) {
      const int mq = t / K, k = t - mq * K;
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
      uint32_t cv = 0, one = 0;
      if (m < M) {
        const uint32_t p = __ldg(b.primes + jb.dst_gidx[m]);
        uint32_t sum = 0;
        for (int k = 0; k < K; k++) {
          const int32_t tv = __ldg(jb.table + m * K + k);
          sum = add_mod(sum, tv < 0 ? static_cast<uint32_t>(tv + static_cast<int32_t>(p)) : static_cast<uint32_t>(tv),
                        p);
        }
        for (int s = 0; s < 30; s++) {  // 2^30 * sum mod p
          sum <<= 1;
          sum = sum >= p ? sum - p : sum;
        }
        cv = sum ? p - sum : 0u;
        one = 0xffffffffu / p;  // p odd: equals floor(2^32 / p)
      }
      corr[buf * 4 + t] = cv;
      ones[buf * 4 + t] = one;
    }
  };

  // one thread: the MMAs of half a chunk (slots 8 half .. 8 half + 7), then commit
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
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem + acc_col(e)),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
  };

  // ---- phase A: INTT column stages, output constant, centring, offset; A
  // rows written four sources (16 bytes) at a time
  for (int kg = 0; kg < K; kg += 4) {
    uint32_t xw[4][8];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int k = kg + kk;
      if (k < K) {
        const int g = jb.src_gidx[k];
        const uint32_t q = __ldg(b.primes + g);
        const uint2 *itw = b.itw + (static_cast<size_t>(g) << 16);
        const uint32_t *src = jb.src + (static_cast<size_t>(jb.src_row[k]) << 16);
        uint32_t y[8];
#pragma unroll
        for (int u = 0; u < 8; u++) y[u] = __ldg(src + (8 * j1 + u) * 512 + col);
        radix8_inv(y, itw, 16 + j1, 32 + 2 * j1, 64 + 4 * j1, q);  // m = 64, 32, 16
#pragma unroll
        for (int u = 0; u < 8; u++) ex[xsw(8 * j1 + u, cl)] = y[u];
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 8; e++) y[e] = ex[xsw(w + 8 * e + 64 * hb, cl)];
        radix8_inv(y, itw, 2 + hb, 4 + 2 * hb, 8 + 4 * hb, q);  // m = 8, 4, 2
        // m = 1 across the lane halves with the output constant:
        // row r <- (a + b) c0, row r + 64 <- (a - b) w1 c0
        const uint32_t cv = hb ? c0w[k].x : jb.c0[k], cs = hb ? c0w[k].y : jb.c0s[k];
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const uint32_t x = reduce2q(y[e], q);
          const uint32_t o = __shfl_xor_sync(0xffffffffu, x, 16);
          const uint32_t d = hb ? o - x + q : x + o;
          const int32_t xc = centre(reduce2q(shoup_lazy(d, cv, cs, q), q), q);
          xw[kk][e] = static_cast<uint32_t>(xc + kOffset);
        }
        __syncthreads();
      } else {
#pragma unroll
        for (int e = 0; e < 8; e++) xw[kk][e] = 0u;
      }
    }
    const int s = kg >> 3, bo = 4 * (kg & 7);
    const int roff = s < G::kFull ? s * 4096 + (R >> 3) * 256 + (bo >> 4) * 128 + (R & 7) * 16 : s * 4096 + R * 16;
#pragma unroll
    for (int e = 0; e < 8; e++)
      *reinterpret_cast<uint4 *>(sa + (2 * e + g2) * G::kSlotBytes + roff) =
          make_uint4(xw[0][e], xw[1][e], xw[2][e], xw[3][e]);
  }
  build_b(0, 0);
  // make the generic-proxy stores visible to the tensor core
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (t == 0) issue(0, 0);

  // ---- phase B: per chunk of 4 targets, TMEM -> residues -> NTT column
  // stages -> HBM
  // stage m = 1 across the lane halves, then m = 2, 4, 8 in registers
  auto front = [&](uint32_t (&x)[8], const uint2 *tw, uint32_t p, uint32_t one) {
    const uint2 w1 = __ldg(tw + 1);
    const uint32_t wv = hb ? w1.x : 1u, ws = hb ? w1.y : one;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const uint32_t mm = reduce2q(shoup_lazy(x[e], wv, ws, p), p);  // a, or w1 b
      const uint32_t o = __shfl_xor_sync(0xffffffffu, mm, 16);
      x[e] = hb ? o - mm + p : mm + o;
    }
    radix8_fwd(x, tw, 2 + hb, 4 + 2 * hb, 8 + 4 * hb, p);
  };
  // stages m = 16, 32, 64 in layout 1, then the store
  auto finish = [&](int m, const uint32_t (&x)[8], const uint2 *tw, uint32_t p) {
#pragma unroll
    for (int e = 0; e < 8; e++) ex[xsw(w + 8 * e + 64 * hb, cl)] = x[e];
    __syncthreads();
    uint32_t *dst = jb.dst + (static_cast<size_t>(jb.dst_row[m]) << 16);
    uint32_t y[8];
#pragma unroll
    for (int u = 0; u < 8; u++) y[u] = ex[xsw(8 * j1 + u, cl)];
    radix8_fwd(y, tw, 16 + j1, 32 + 2 * j1, 64 + 4 * j1, p);
#pragma unroll
    for (int u = 0; u < 8; u++) dst[(8 * j1 + u) * 512 + col] = y[u];
    __syncthreads();
  };
  uint32_t phase = 0;
  bool ok = true;
  for (int c = 0; c < nch && ok; c++) {
    const int buf = c & 1;
    uint32_t p[4], one[4];
    int32_t pinv[4];
    uint32_t v[4][8];
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
#pragma unroll
      for (int mq = 0; mq < 4; mq++) {
        const int m = 4 * c + mq;
        const int g = m < M ? jb.dst_gidx[m] : 0;
        p[mq] = m < M ? __ldg(b.primes + g) : 1u;
        pinv[mq] = m < M ? __ldg(b.qinvs + g) : 1;
        cr[mq] = corr[buf * 4 + mq];
        one[mq] = ones[buf * 4 + mq];
      }
#pragma unroll
      for (int i = 0; i < 4; i += 2) {
        uint32_t r[32];
        tmem_ld32(tmem + lane_base + 64u * g2 + 16u * i, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int mq = 0; mq < 4; mq++) {
            const uint32_t *d = r + 16 * h + 4 * mq;
            const uint32_t lo = d[0] + (d[1] << 8) + cr[mq];
            const uint32_t hi = d[2] + (d[3] << 8);
            const uint64_t val = (static_cast<uint64_t>(hi) << 16) + lo;
            v[mq][4 * half + i + h] = mont_reduce(static_cast<int64_t>(val), p[mq], pinv[mq]);
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
        front(v[mq], tw0, p[mq], one[mq]);
        front(v[mq + 1], tw1, p[mq + 1], one[mq + 1]);
        finish(m, v[mq], tw0, p[mq]);
        finish(m + 1, v[mq + 1], tw1, p[mq + 1]);
      } else if (m < M) {
        const uint2 *tw0 = b.tw + (static_cast<size_t>(jb.dst_gidx[m]) << 16);
        front(v[mq], tw0, p[mq], one[mq]);
        finish(m, v[mq], tw0, p[mq]);
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

template <int KMAX, int MINB>
void launch_kmax8(const MSColBatch &b, cudaStream_t s) {
  // CTAs per SM: up to 3 for KMAX = 8 (shared memory), 2 for 12; their
  // accumulators (128 TMEM columns each) always fit
  const size_t sm = Geo8<KMAX>::kSmem;
  cudaFuncSetAttribute(k_modswitch_cols_tc8<KMAX, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(sm));
  k_modswitch_cols_tc8<KMAX, MINB><<<dim3(512 / kTC, b.count), kThreads, sm, s>>>(b);
}

}  // namespace

bool modswitch_cols_tc8_supports(int max_k) { return max_k >= 1 && max_k <= 12; }

void launch_modswitch_cols_tc8(const MSColBatch &b, int max_k, bool regs128, cudaStream_t s) {
  if (b.count <= 0) return;
  if (max_k <= 8) {
    if (regs128)
      launch_kmax8<8, 2>(b, s);
    else
      launch_kmax8<8, 3>(b, s);
  } else {
    launch_kmax8<12, 2>(b, s);
  }
}

}  // namespace chd
