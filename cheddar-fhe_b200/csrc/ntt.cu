// Negacyclic NTT / INTT kernels.
//
// Transform semantics (what every kernel here must reproduce exactly): the
// forward transform of a limb a (natural order) is
//     A[k] = sum_i a_i * psi^((2 brev(k) + 1) i)  mod q,
// stored bit-reversed, with psi the primitive 2N-th root derived from the
// smallest generator of Z_q^* and twiddles psi_rev[j] = psi^brev(j)
// (src/core/NTT.cu:1233-1299 and include/common/PrimeUtils.h:135-196 of the
// reference).  Stage m of the Cooley-Tukey network pairs index j with
// j + N/(2m) using twiddle psi_rev[m + floor(j m / N)]; the inverse runs the
// Gentleman-Sande network with psi^-1.  All arithmetic is exact mod q: values
// travel lazily in [0, 2q) between stages (Shoup products, arith.cuh) and are
// reduced to [0, q) on output, so every output word is the canonical residue.
//
// Layout for N = 2^16: the limb is a 128 x 512 row-major matrix.  Stages
// m = 1..64 only pair elements of the same column (128-point column
// transforms, one CTA per 32-column tile, shared twiddles); stages
// m = 128..32768 stay inside one 512-element row (one CTA per 4 rows, three
// radix-8 rounds exchanged through shared memory).  The inverse runs rows
// first, then columns, and fuses the per-limb output constant and the
// optional centring into the column phase.  For N <= 2^15 the whole limb
// fits in shared memory and one kernel runs every stage.
#include "arith.cuh"
#include "kernels.h"
#include "ntt_common.cuh"

namespace chd {
namespace {

constexpr int kColTile = 32;

// ---------------------------------------------------------------- N = 2^16
__global__ void __launch_bounds__(256) k_fwd_cols16(const __grid_constant__ RowBatch rb) {
  __shared__ uint32_t sm[128 * kColTile];
  const RowDesc &rd = rb.rows[blockIdx.y];
  const uint32_t q = rd.q;
  const uint2 *tw = rd.tw;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * kColTile + lane;
  uint32_t x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = __ldg(rd.src + (w + 8 * k) * 512 + c);
  if (rd.flags & kPreMult) {
#pragma unroll
    for (int k = 0; k < 16; k++) x[k] = shoup_lazy(x[k], rd.c0, rd.c0s, q);
  }
  radix16_cols_fwd(x, tw, q);  // stages m = 1, 2, 4, 8 on rows w + 8k
#pragma unroll
  for (int k = 0; k < 16; k++) sm[(w + 8 * k) * kColTile + lane] = x[k];
  __syncthreads();
  // stages m = 16, 32, 64 on rows 8j + u (j = 2w + hh)
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int j = 2 * w + hh;
    uint32_t y[8];
#pragma unroll
    for (int u = 0; u < 8; u++) y[u] = sm[(8 * j + u) * kColTile + lane];
    radix8_fwd(y, tw, 16 + j, 32 + 2 * j, 64 + 4 * j, q);
#pragma unroll
    for (int u = 0; u < 8; u++) rd.dst[(8 * j + u) * 512 + c] = y[u];  // lazy [0, 2q)
  }
}

// Row phase of the forward transform (input lazy from the column phase),
// canonical output, with the optional ModDown epilogue (src2 * c1 - x) * c2.
__global__ void __launch_bounds__(256) k_fwd_rows16(const __grid_constant__ RowBatch rb) {
  __shared__ uint32_t sm[4][512];
  const RowDesc &rd = rb.rows[blockIdx.y];
  const uint32_t q = rd.q;
  const uint2 *tw = rd.tw;
  const int t = threadIdx.x & 63, rl = threadIdx.x >> 6;
  const int r = blockIdx.x * 4 + rl;
  uint32_t *srow = sm[rl];
  const uint32_t *src = rd.dst + r * 512;  // the column phase wrote dst
  uint32_t x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = src[t + 64 * k];
  row_fwd(x, srow, tw, r, t, q, -1);
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = reduce2q(x[k], q);
  const int base = r * 512 + 8 * t;
  if (rd.flags & kModDownEpi) {
    uint32_t v[8];
    if (rd.flags & kHasSrc2) {
      const uint4 *p2 = reinterpret_cast<const uint4 *>(rd.src2 + base);
      uint4 a0 = __ldg(p2), a1 = __ldg(p2 + 1);
      v[0] = a0.x; v[1] = a0.y; v[2] = a0.z; v[3] = a0.w;
      v[4] = a1.x; v[5] = a1.y; v[6] = a1.z; v[7] = a1.w;
      if (rd.flags & kPadSrc2) {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = reduce2q(shoup_lazy(v[k], rd.c1, rd.c1s, q), q);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = reduce2q(shoup_lazy(v[k] - x[k] + q, rd.c2, rd.c2s, q), q);
  }
  uint4 *o = reinterpret_cast<uint4 *>(rd.dst + base);
  o[0] = make_uint4(x[0], x[1], x[2], x[3]);
  o[1] = make_uint4(x[4], x[5], x[6], x[7]);
}

// Inverse, row phase: Gentleman-Sande stages m = 32768 .. 128 (lazy output).
__global__ void __launch_bounds__(256) k_inv_rows16(const __grid_constant__ RowBatch rb) {
  __shared__ uint32_t sm[4][512];
  const RowDesc &rd = rb.rows[blockIdx.y];
  const uint32_t q = rd.q;
  const uint2 *tw = rd.tw;
  const int t = threadIdx.x & 63, rl = threadIdx.x >> 6;
  const int r = blockIdx.x * 4 + rl;
  uint32_t *srow = sm[rl];
  const int base = r * 512 + 8 * t;
  uint32_t x[8];
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(rd.src + base);
    uint4 a0 = __ldg(p), a1 = __ldg(p + 1);
    x[0] = a0.x; x[1] = a0.y; x[2] = a0.z; x[3] = a0.w;
    x[4] = a1.x; x[5] = a1.y; x[6] = a1.z; x[7] = a1.w;
  }
  if (rd.flags & kMulSrc2) {
    const uint4 *p = reinterpret_cast<const uint4 *>(rd.src2 + base);
    uint4 a0 = __ldg(p), a1 = __ldg(p + 1);
    const uint32_t y[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = mont_mul(x[k], y[k], q, rd.qinv);
  }
  row_inv(x, srow, tw, r, t, q, -1);
  uint32_t *dst = rd.dst + r * 512;
#pragma unroll
  for (int k = 0; k < 8; k++) dst[t + 64 * k] = x[k];
}

// Inverse, column phase: stages m = 64 .. 1, then x * c0, canonical or centred.
__global__ void __launch_bounds__(256) k_inv_cols16(const __grid_constant__ RowBatch rb) {
  __shared__ uint32_t sm[128 * kColTile];
  const RowDesc &rd = rb.rows[blockIdx.y];
  const uint32_t q = rd.q;
  const uint2 *tw = rd.tw;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * kColTile + lane;
  const uint32_t *src = rd.dst;  // the row phase wrote dst
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int j = 2 * w + hh;
    uint32_t y[8];
#pragma unroll
    for (int u = 0; u < 8; u++) y[u] = src[(8 * j + u) * 512 + c];
    radix8_inv(y, tw, 16 + j, 32 + 2 * j, 64 + 4 * j, q);
#pragma unroll
    for (int u = 0; u < 8; u++) sm[(8 * j + u) * kColTile + lane] = y[u];
  }
  __syncthreads();
  uint32_t x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = sm[(w + 8 * k) * kColTile + lane];
  radix16_cols_inv(x, tw, q);  // stages m = 8, 4, 2, 1 on rows w + 8k
  const bool centre_out = (rd.flags & kCentre) != 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    uint32_t v = reduce2q(shoup_lazy(x[k], rd.c0, rd.c0s, q), q);
    if (centre_out) v = static_cast<uint32_t>(centre(v, q));
    rd.dst[(w + 8 * k) * 512 + c] = v;
  }
}

// ------------------------------------------------------------ N <= 2^15
// Whole limb in shared memory, one CTA per limb.
template <bool kFwd>
__global__ void __launch_bounds__(1024) k_small(const __grid_constant__ RowBatch rb, int log_n) {
  extern __shared__ uint32_t sa[];
  const RowDesc &rd = rb.rows[blockIdx.x];
  const uint32_t q = rd.q;
  const uint2 *tw = rd.tw;
  const int n = 1 << log_n, half = n >> 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t v = rd.src[i];
    if (kFwd && (rd.flags & kPreMult)) v = shoup_lazy(v, rd.c0, rd.c0s, q);
    sa[i] = v;
  }
  __syncthreads();
  if (kFwd) {
    for (int m = 1, lt = log_n - 1; m < n; m <<= 1, lt--) {
      const int t = 1 << lt;
      for (int b = threadIdx.x; b < half; b += blockDim.x) {
        const int i = b >> lt, j = 2 * i * t + (b & (t - 1));
        ct_lazy(sa[j], sa[j + t], __ldg(tw + m + i), q);
      }
      __syncthreads();
    }
  } else {
    for (int m = half, lt = 0; m >= 1; m >>= 1, lt++) {
      const int t = 1 << lt;
      for (int b = threadIdx.x; b < half; b += blockDim.x) {
        const int i = b >> lt, j = 2 * i * t + (b & (t - 1));
        gs_lazy(sa[j], sa[j + t], __ldg(tw + m + i), q);
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t x = reduce2q(sa[i], q);
    if (kFwd) {
      if (rd.flags & kModDownEpi) {
        uint32_t v = 0;
        if (rd.flags & kHasSrc2) {
          v = rd.src2[i];
          if (rd.flags & kPadSrc2) v = reduce2q(shoup_lazy(v, rd.c1, rd.c1s, q), q);
        }
        x = reduce2q(shoup_lazy(v - x + q, rd.c2, rd.c2s, q), q);
      }
    } else {
      x = reduce2q(shoup_lazy(x, rd.c0, rd.c0s, q), q);
      if (rd.flags & kCentre) x = static_cast<uint32_t>(centre(x, q));
    }
    rd.dst[i] = x;
  }
}

}  // namespace

void launch_ntt_fwd_cols(const RowBatch &rb, int log_n, cudaStream_t s) {
  if (rb.count <= 0) return;
  k_fwd_cols16<<<dim3(512 / kColTile, rb.count), 256, 0, s>>>(rb);
}

void launch_ntt_fwd_rows(const RowBatch &rb, int log_n, cudaStream_t s) {
  if (rb.count <= 0) return;
  k_fwd_rows16<<<dim3(128 / 4, rb.count), 256, 0, s>>>(rb);
}

void launch_ntt_fwd(const RowBatch &rb, int log_n, cudaStream_t s) {
  if (rb.count <= 0) return;
  if (log_n == 16) {
    launch_ntt_fwd_cols(rb, log_n, s);
    launch_ntt_fwd_rows(rb, log_n, s);
  } else {
    size_t smem = sizeof(uint32_t) << log_n;
    cudaFuncSetAttribute(k_small<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024);
    k_small<true><<<rb.count, 1024, smem, s>>>(rb, log_n);
  }
}

void launch_ntt_inv_rows(const RowBatch &rb, int log_n, cudaStream_t s) {
  if (rb.count <= 0) return;
  k_inv_rows16<<<dim3(128 / 4, rb.count), 256, 0, s>>>(rb);
}

void launch_ntt_inv(const RowBatch &rb, int log_n, cudaStream_t s) {
  if (rb.count <= 0) return;
  if (log_n == 16) {
    k_inv_rows16<<<dim3(128 / 4, rb.count), 256, 0, s>>>(rb);
    k_inv_cols16<<<dim3(512 / kColTile, rb.count), 256, 0, s>>>(rb);
  } else {
    size_t smem = sizeof(uint32_t) << log_n;
    cudaFuncSetAttribute(k_small<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024);
    k_small<false><<<rb.count, 1024, smem, s>>>(rb, log_n);
  }
}

}  // namespace chd
