// Base conversion on the tcgen05 tensor cores (INT8 limb split, exact).
//
// BConv (kernel::ModSwitchMatrixMult, src/core/ModSwitch.cu:23-171 of the
// reference) computes, per coefficient n and target prime p_m,
//   out[m][n] = (sum_k x_k[n] * T[m][k]) * 2^-32 mod p_m
// with centred sources |x_k| < 2^30 and the centred table T (k_bconv in
// elem.cu does it with int64 multiply-adds).  Here the contraction runs as an
// int8 GEMM with int32 accumulation:
//   * each source is split into four balanced signed bytes,
//     x = sum_j 2^(8j) s_j, s_j in [-128, 127]   (A operand, s8, [coeff][4K]);
//   * each constant c[m][k][j] = 2^(8j) T[m][k] mod p_m (canonical, < 2^31) is
//     split into four unsigned bytes u[m][k][j][i]  (B operand, u8, [4M][4K]);
//   * D[n][4m+i] = sum_(k,j) s_j(x_k[n]) u[m][k][j][i]  (|D| < 2^21 for K <= 16)
//     is exact in int32, and V = sum_i 2^(8i) D[n][4m+i] (|V| < 2^46) is
//     congruent to sum_k x_k T[m][k] mod p_m.
// The Montgomery reduction of V therefore yields the same canonical residue
// as the int64 path: the output is bit-identical.
//
// One CTA (4 warps, thread t <-> coefficient row t of a 128-row tile) loops
// over tiles: sources -> balanced bytes -> shared memory in the canonical
// K-major no-swizzle layout -> one thread issues the MMAs (M = 128,
// N = 4M padded to 16, K = 32 bytes per instruction) into TMEM and commits
// them to an mbarrier -> every warp reads its 32 TMEM lanes back and
// recombines.  The B operand is prepared once per call on the host in the
// same layout and copied linearly into shared memory.
#include <algorithm>

#include "arith.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace chd {
namespace {

using namespace tc;

constexpr int kRows = 128;          // coefficients per tile (MMA M)
constexpr int kATileBytes = kRows * 32;  // one K-step of A: 128 rows x 32 bytes
// balanced base-256 digits of a centred residue, packed little-endian
__device__ __forceinline__ uint32_t split_s8(int32_t x) {
  const int32_t s0 = static_cast<int8_t>(x & 0xff);
  x = (x - s0) >> 8;
  const int32_t s1 = static_cast<int8_t>(x & 0xff);
  x = (x - s1) >> 8;
  const int32_t s2 = static_cast<int8_t>(x & 0xff);
  x = (x - s2) >> 8;  // |x| <= 65 for |input| < 2^30
  return (static_cast<uint32_t>(s0) & 0xff) | ((static_cast<uint32_t>(s1) & 0xff) << 8) |
         ((static_cast<uint32_t>(s2) & 0xff) << 16) | (static_cast<uint32_t>(x) << 24);
}

// Software pipeline over iterations (TPI tiles each), two buffers for the A
// tiles and the TMEM accumulators:
//   split + store A(i) -> MMA(i) -> loads of i+DEPTH in flight -> epilogue(i-1)
// so the HBM loads of the next DEPTH iterations overlap the MMAs of the
// current one and the TMEM read-back and stores of the previous one.  The
// loads sit in a ring of DEPTH register stages: with few sources per tile
// (a ModDown from 4 auxiliary primes: 16 bytes per thread and tile) one
// stage keeps too few bytes in flight for HBM, and the TMEM columns that the
// targets' accumulators take cap the CTAs per SM.
template <int TPI, int KMAX>
struct BConvTcShape {
  static constexpr int kDepth = TPI * KMAX <= 8 ? 4 : (TPI * KMAX <= 16 ? 2 : 1);
};

template <int TPI, int KMAX>
__global__ void __launch_bounds__(128) k_bconv_tc(const __grid_constant__ BConvTcDesc d) {
  constexpr int DEPTH = BConvTcShape<TPI, KMAX>::kDepth;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[3];  // two accumulator buffers + the stall-test barrier
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, w = t >> 5;
  const int KS = d.ksteps, NB = d.nb, K = d.K, M = d.M;
  const int abuf = TPI * KS * kATileBytes;            // one A buffer
  uint8_t *sa = smem;                                 // 2 x TPI x KS x 4096 bytes
  uint8_t *sb = smem + 2 * abuf;                      // KS x NB x 32 bytes
  const uint32_t sa_u = smem_u32(sa), sb_u = smem_u32(sb);
  const uint32_t bar0 = smem_u32(&mbar[0]), bar1 = smem_u32(&mbar[1]);
  const uint32_t bar_never = smem_u32(&mbar[2]);  // initialised, never arrived at

  // B operand: already in the canonical layout, copy linearly
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(d.bmat);
    uint4 *dst = reinterpret_cast<uint4 *>(sb);
    for (int i = t; i < KS * NB * 2; i += 128) dst[i] = src[i];
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_never) : "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(d.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = static_cast<uint32_t>(32 * (w & 3)) << 16;
  const uint32_t tbuf = static_cast<uint32_t>(TPI * NB);  // TMEM columns of one accumulator buffer

  // an iteration takes TPI consecutive 128-row tiles of one polynomial
  // (TPI divides the tiles per polynomial)
  const int tiles_per_poly = d.n / kRows;
  const int nits = d.npoly * tiles_per_poly / TPI;
  const size_t n = static_cast<size_t>(d.n);
  auto src_of = [&](int it) {
    const int tile0 = it * TPI;
    return d.xt + static_cast<size_t>(tile0 / tiles_per_poly) * K * n +
           static_cast<size_t>(tile0 % tiles_per_poly) * kRows + t;
  };
  auto dst_of = [&](int it) {
    const int tile0 = it * TPI;
    return d.out + static_cast<size_t>(tile0 / tiles_per_poly) * M * n +
           static_cast<size_t>(tile0 % tiles_per_poly) * kRows + t;
  };
  int32_t v[DEPTH][TPI][KMAX];
  auto load = [&](int32_t (&dst)[TPI][KMAX], int it) {
    const int32_t *x = src_of(it);
#pragma unroll
    for (int u = 0; u < TPI; u++)
#pragma unroll
      for (int k = 0; k < KMAX; k++) dst[u][k] = k < K ? __ldg(x + static_cast<size_t>(k) * n + u * kRows) : 0;
  };
  auto epilogue = [&](int it, int b) {
    uint32_t *o = dst_of(it);
#pragma unroll
    for (int u = 0; u < TPI; u++)
      for (int m0 = 0; m0 < M; m0 += 4) {
        uint32_t r[16];
        tmem_ld16(tmem + lane_base + b * tbuf + static_cast<uint32_t>(u * NB + 4 * m0), r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int m = m0 + e;
          if (m < M) {
            const int64_t val = static_cast<int64_t>(static_cast<int32_t>(r[4 * e])) +
                                (static_cast<int64_t>(static_cast<int32_t>(r[4 * e + 1])) << 8) +
                                (static_cast<int64_t>(static_cast<int32_t>(r[4 * e + 2])) << 16) +
                                (static_cast<int64_t>(static_cast<int32_t>(r[4 * e + 3])) << 24);
            o[static_cast<size_t>(m) * n + u * kRows] = mont_reduce(val, d.p[m], d.pinv[m]);
          }
        }
      }
  };

  // phase parity of each accumulator buffer's mbarrier (bit b), kept in a
  // register
  uint32_t parity = 0u;
  uint32_t pending = 0u;  // accumulator buffers with committed MMAs not yet waited for
  bool ok = true;
  int prev = -1;  // iteration whose accumulators wait for their epilogue
  int it = blockIdx.x;
  const int grid = static_cast<int>(gridDim.x);
#pragma unroll
  for (int s = 0; s < DEPTH; s++)
    if (it + s * grid < nits) load(v[s], it + s * grid);
  int i = 0;
  while (ok && it < nits) {
    // the ring is walked with compile-time stage indices (registers)
#pragma unroll
    for (int st = 0; st < DEPTH; st++) {
      if (!ok || it >= nits) continue;
      const int b = i & 1;
      // A operand of tile u: row t, chunk c (sources 4c..4c+3) at
      //   b * abuf + (u * KS + c / 2) * 4096 + (t / 8) * 256 + (c % 2) * 128 + (t % 8) * 16
#pragma unroll
      for (int u = 0; u < TPI; u++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if (c < 2 * KS) {
            uint32_t wd[4];
#pragma unroll
            for (int j = 0; j < 4; j++) wd[j] = 4 * c + j < KMAX ? split_s8(v[st][u][(4 * c + j) % KMAX]) : 0u;
            const int off =
                b * abuf + (u * KS + (c >> 1)) * kATileBytes + (t >> 3) * 256 + (c & 1) * 128 + (t & 7) * 16;
            *reinterpret_cast<uint4 *>(sa + off) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
          }
        }
      // make the generic-proxy stores visible to the tensor core
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int u = 0; u < TPI; u++)
          for (int s = 0; s < KS; s++) {
            const uint64_t ad = smem_desc(sa_u + b * abuf + (u * KS + s) * kATileBytes, 128, 256);
            const uint64_t bd = smem_desc(sb_u + s * NB * 32, 128, 256);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                ::"r"(tmem + b * tbuf + static_cast<uint32_t>(u * NB)), "l"(ad), "l"(bd), "r"(d.idesc), "r"(acc),
                "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                : "memory");
          }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(b ? bar1
                                                                                                            : bar0)
                     : "memory");
      }
      pending |= 1u << b;
      // this stage's next loads (DEPTH iterations ahead) go out while the MMAs run
      if (it + DEPTH * grid < nits) load(v[st], it + DEPTH * grid);
      if (prev >= 0) {
        const int pb = b ^ 1;
        // every thread polls with a limit; the CTA leaves together if any gave up
        const bool got = d.stall_polls ? mbar_wait(bar_never, 0u, d.stall_polls)
                                       : mbar_wait(pb ? bar1 : bar0, (parity >> pb) & 1u);
        if (!__syncthreads_and(got ? 1 : 0)) {
          ok = false;
          continue;
        }
        parity ^= 1u << pb;
        pending &= ~(1u << pb);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        epilogue(prev, pb);
        // TMEM reads of buffer pb finish before MMAs overwrite it
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
      prev = it;
      i++;
      it += grid;
    }
  }
  if (ok && prev >= 0) {
    // the last iteration's accumulators sit in buffer ((iterations - 1) & 1)
    const int nmine = (nits - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1;
    const int pb = (nmine - 1) & 1;
    const bool got = d.stall_polls ? mbar_wait(bar_never, 0u, d.stall_polls)
                                   : mbar_wait(pb ? bar1 : bar0, (parity >> pb) & 1u);
    if (__syncthreads_and(got ? 1 : 0)) {
      parity ^= 1u << pb;
      pending &= ~(1u << pb);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(prev, pb);
    } else {
      ok = false;
    }
  }
  if (!ok) {
    if (t == 0 && d.err) atomicExch(d.err, 1);
    // give the MMAs in flight (committed, not yet waited for) a second
    // bounded chance to land before TMEM is freed
    if (pending & 1u) mbar_wait(bar0, parity & 1u);
    if (pending & 2u) mbar_wait(bar1, (parity >> 1) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (w == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(d.tmem_cols) : "memory");
  }
}

}  // namespace

size_t bconv_tc_smem(int tpi, int ksteps, int nb) {
  return static_cast<size_t>(ksteps) * (2 * static_cast<size_t>(tpi) * kATileBytes + nb * 32);
}

namespace {
template <int TPI, int KMAX>
int launch_tpi(const BConvTcDesc &d, int num_sms, cudaStream_t s) {
  // CTAs per SM: TMEM (512 columns), registers, shared memory (228 KiB per
  // SM, 1 KiB reserved per CTA), 16 CTAs of 128 threads; the dynamic shared
  // memory is padded so that no more CTAs than the TMEM allows are resident
  const int cap = 512 / d.tmem_cols;
  size_t sm = bconv_tc_smem(TPI, d.ksteps, d.nb);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, k_bconv_tc<TPI, KMAX>) != cudaSuccess) return -2;
  const size_t per_sm = 233472, reserved = 1024 + fa.sharedSizeBytes;
  const size_t floor_sm = per_sm / (cap + 1) + 16 > reserved ? per_sm / (cap + 1) + 16 - reserved : 0;
  if (sm < floor_sm) sm = floor_sm;
  if (cudaFuncSetAttribute(k_bconv_tc<TPI, KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(sm)) != cudaSuccess)
    return -2;
  int per = cap;
  const int regs = fa.numRegs > 0 ? fa.numRegs : 64;
  per = std::min(per, 65536 / (regs * 128));
  per = std::min(per, static_cast<int>(per_sm / (sm + reserved)));
  per = std::min(per, 16);
  if (per < 1) return -2;
  const int nits = d.npoly * (d.n / kRows) / TPI;
  int grid = num_sms * per;
  if (grid > nits) grid = nits;
  k_bconv_tc<TPI, KMAX><<<grid, 128, sm, s>>>(d);
  return 0;
}

template <int TPI>
int launch_kmax(const BConvTcDesc &d, int num_sms, cudaStream_t s) {
  if (d.K <= 4) return launch_tpi<TPI, 4>(d, num_sms, s);
  if (d.K <= 8) return launch_tpi<TPI, 8>(d, num_sms, s);
  if (d.K <= 12) return launch_tpi<TPI, 12>(d, num_sms, s);
  return launch_tpi<TPI, 16>(d, num_sms, s);
}
}  // namespace

int launch_bconv_tc(const BConvTcDesc &d, int num_sms, cudaStream_t s) {
  if (d.npoly <= 0) return 0;
  if (d.n % kRows != 0 || d.K < 1 || d.K > 16 || d.M < 1 || d.M > 64 || 2 * d.tpi * d.nb > d.tmem_cols ||
      d.tmem_cols > 512)
    return -1;
  if ((d.n / kRows) % d.tpi != 0) return -1;
  switch (d.tpi) {
    case 1: return launch_kmax<1>(d, num_sms, s);
    case 2: return launch_kmax<2>(d, num_sms, s);
    case 4: return launch_kmax<4>(d, num_sms, s);
    default: return -1;
  }
}

}  // namespace chd
