// Kernels of the 64-bit word path (w64.h), N = 2^16: the NTT in two passes
// (column stages on 128 x 32 tiles, row stages on 512-element rows, the
// layout and twiddle semantics of the 32-bit path), exact base conversion
// with 128-bit accumulation, tensor product, key inner product and the
// automorphism.  Lazy Shoup butterflies keep values in [0, 2q) (q < 2^62);
// Montgomery products use R = 2^64 as the reference's
// __mult_montgomery_lazy<uint64_t> (include/common/Basic.cuh:128-137).
#include "w64.h"

namespace chd {
namespace w64 {
namespace {

constexpr int kColTile = 32;

__device__ __forceinline__ u64 shoup(u64 b, u64 w, u64 ws, u64 q) { return b * w - __umul64hi(b, ws) * q; }
__device__ __forceinline__ u64 red2q(u64 x, u64 q) { return x >= q ? x - q : x; }
__device__ __forceinline__ u64 add_mod(u64 a, u64 b, u64 q) { return red2q(a + b, q); }
// Montgomery reduction of a signed 128-bit value (|a| < q 2^63): a 2^-64 mod q
__device__ __forceinline__ u64 redc(i128 a, u64 q, i64 qinv) {
  const i64 lo = static_cast<i64>(a), hi = static_cast<i64>(a >> 64);
  const i64 t = lo * qinv;
  i64 r = hi - __mul64hi(t, static_cast<i64>(q));
  if (r < 0) r += static_cast<i64>(q);
  return static_cast<u64>(r);
}
__device__ __forceinline__ u64 mont_mul(u64 a, u64 b, u64 q, i64 qinv) {
  return redc(static_cast<i128>(static_cast<u128>(a) * b), q, qinv);
}
__device__ __forceinline__ i64 centre(u64 a, u64 q) {
  return a > (q >> 1) ? static_cast<i64>(a) - static_cast<i64>(q) : static_cast<i64>(a);
}

// butterflies on lazy [0, 2q) values
__device__ __forceinline__ void ct(u64 &a, u64 &b, ulonglong2 w, u64 q) {
  const u64 x = red2q(a, q);
  const u64 t = red2q(shoup(b, w.x, w.y, q), q);
  a = x + t;
  b = x - t + q;
}
__device__ __forceinline__ void gs(u64 &a, u64 &b, ulonglong2 w, u64 q) {
  const u64 x = red2q(a, q), y = red2q(b, q);
  a = x + y;
  b = shoup(x - y + q, w.x, w.y, q);
}

// radix-8 networks on x[0..7] at register distances 4, 2, 1 (forward) with
// twiddles tw[b0], tw[b1 + g], tw[b2 + g]
__device__ __forceinline__ void r8_fwd(u64 *x, const ulonglong2 *tw, int b0, int b1, int b2, u64 q) {
  const ulonglong2 w0 = tw[b0];
#pragma unroll
  for (int k = 0; k < 4; k++) ct(x[k], x[k + 4], w0, q);
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const ulonglong2 w1 = tw[b1 + g];
    ct(x[4 * g], x[4 * g + 2], w1, q);
    ct(x[4 * g + 1], x[4 * g + 3], w1, q);
  }
#pragma unroll
  for (int g = 0; g < 4; g++) ct(x[2 * g], x[2 * g + 1], tw[b2 + g], q);
}
__device__ __forceinline__ void r8_inv(u64 *x, const ulonglong2 *tw, int b0, int b1, int b2, u64 q) {
#pragma unroll
  for (int g = 0; g < 4; g++) gs(x[2 * g], x[2 * g + 1], tw[b2 + g], q);
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const ulonglong2 w1 = tw[b1 + g];
    gs(x[4 * g], x[4 * g + 2], w1, q);
    gs(x[4 * g + 1], x[4 * g + 3], w1, q);
  }
  const ulonglong2 w0 = tw[b0];
#pragma unroll
  for (int k = 0; k < 4; k++) gs(x[k], x[k + 4], w0, q);
}
// column stages m = 1, 2, 4, 8 on 16 registers holding rows w + 8k
__device__ __forceinline__ void r16_cols_fwd(u64 *x, const ulonglong2 *tw, u64 q) {
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int m = 1 << s, h = 8 >> s;
#pragma unroll
    for (int g = 0; g < m; g++) {
      const ulonglong2 w = tw[m + g];
#pragma unroll
      for (int j = 0; j < h; j++) ct(x[g * 2 * h + j], x[g * 2 * h + j + h], w, q);
    }
  }
}
__device__ __forceinline__ void r16_cols_inv(u64 *x, const ulonglong2 *tw, u64 q) {
#pragma unroll
  for (int s = 3; s >= 0; s--) {
    const int m = 1 << s, h = 8 >> s;
#pragma unroll
    for (int g = 0; g < m; g++) {
      const ulonglong2 w = tw[m + g];
#pragma unroll
      for (int j = 0; j < h; j++) gs(x[g * 2 * h + j], x[g * 2 * h + j + h], w, q);
    }
  }
}

// forward column phase: rows w + 8k (k < 16) of 32 columns per CTA
__global__ void __launch_bounds__(256) k64_fwd_cols(const __grid_constant__ RowBatch64 rb) {
  __shared__ u64 sm[128 * kColTile];
  const Row64 &rd = rb.rows[blockIdx.y];
  const u64 q = rd.q;
  const ulonglong2 *tw = rd.tw;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * kColTile + lane;
  u64 x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = rd.src[(w + 8 * k) * 512 + c];
  if (rd.flags & kPreMult) {
#pragma unroll
    for (int k = 0; k < 16; k++) x[k] = shoup(x[k], rd.c0, rd.c0s, q);
  }
  r16_cols_fwd(x, tw, q);
#pragma unroll
  for (int k = 0; k < 16; k++) sm[(w + 8 * k) * kColTile + lane] = x[k];
  __syncthreads();
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int j = 2 * w + hh;
    u64 y[8];
#pragma unroll
    for (int u = 0; u < 8; u++) y[u] = sm[(8 * j + u) * kColTile + lane];
    r8_fwd(y, tw, 16 + j, 32 + 2 * j, 64 + 4 * j, q);
#pragma unroll
    for (int u = 0; u < 8; u++) rd.dst[(8 * j + u) * 512 + c] = y[u];
  }
}

__device__ __forceinline__ int rsw(int c) { return c ^ ((c >> 3) & 31); }

// forward row phase (9 stages on one 512-element row held by 64 threads),
// canonical output, optional ModDown epilogue (src2 c1 - x) c2
__global__ void __launch_bounds__(256) k64_fwd_rows(const __grid_constant__ RowBatch64 rb) {
  __shared__ u64 sm[4][512];
  const Row64 &rd = rb.rows[blockIdx.y];
  const u64 q = rd.q;
  const ulonglong2 *tw = rd.tw;
  const int t = threadIdx.x & 63, rl = threadIdx.x >> 6;
  const int r = blockIdx.x * 4 + rl;
  u64 *srow = sm[rl];
  const u64 *src = rd.dst + r * 512;
  const int b = t >> 3, u0 = t & 7;
  u64 x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = src[t + 64 * k];
  r8_fwd(x, tw, 128 + r, 256 + 2 * r, 512 + 4 * r, q);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(t + 64 * k)] = x[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(64 * b + u0 + 8 * k)];
  r8_fwd(x, tw, 1024 + 8 * r + b, 2048 + 16 * r + 2 * b, 4096 + 32 * r + 4 * b, q);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(64 * b + u0 + 8 * k)] = x[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(8 * t + k)];
  r8_fwd(x, tw, 8192 + 64 * r + t, 16384 + 128 * r + 2 * t, 32768 + 256 * r + 4 * t, q);
  const int base = r * 512 + 8 * t;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    u64 v = red2q(x[k], q);
    if (rd.flags & kModDownEpi) {
      u64 s2 = 0;
      if (rd.flags & kHasSrc2) {
        s2 = rd.src2[base + k];
        if (rd.flags & kPadSrc2) s2 = red2q(shoup(s2, rd.c1, rd.c1s, q), q);
      }
      v = red2q(shoup(s2 - v + q, rd.c2, rd.c2s, q), q);
    }
    rd.dst[base + k] = v;
  }
}

// inverse row phase (lazy output)
__global__ void __launch_bounds__(256) k64_inv_rows(const __grid_constant__ RowBatch64 rb) {
  __shared__ u64 sm[4][512];
  const Row64 &rd = rb.rows[blockIdx.y];
  const u64 q = rd.q;
  const ulonglong2 *tw = rd.tw;
  const int t = threadIdx.x & 63, rl = threadIdx.x >> 6;
  const int r = blockIdx.x * 4 + rl;
  u64 *srow = sm[rl];
  const int b = t >> 3, u0 = t & 7;
  const int base = r * 512 + 8 * t;
  u64 x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = rd.src[base + k];
  r8_inv(x, tw, 8192 + 64 * r + t, 16384 + 128 * r + 2 * t, 32768 + 256 * r + 4 * t, q);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(8 * t + k)] = x[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(64 * b + u0 + 8 * k)];
  r8_inv(x, tw, 1024 + 8 * r + b, 2048 + 16 * r + 2 * b, 4096 + 32 * r + 4 * b, q);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(64 * b + u0 + 8 * k)] = x[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(t + 64 * k)];
  r8_inv(x, tw, 128 + r, 256 + 2 * r, 512 + 4 * r, q);
  u64 *dst = rd.dst + r * 512;
#pragma unroll
  for (int k = 0; k < 8; k++) dst[t + 64 * k] = x[k];
}

// inverse column phase, then x c0, canonical or centred
__global__ void __launch_bounds__(256) k64_inv_cols(const __grid_constant__ RowBatch64 rb) {
  __shared__ u64 sm[128 * kColTile];
  const Row64 &rd = rb.rows[blockIdx.y];
  const u64 q = rd.q;
  const ulonglong2 *tw = rd.tw;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * kColTile + lane;
  const u64 *src = rd.dst;
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int j = 2 * w + hh;
    u64 y[8];
#pragma unroll
    for (int u = 0; u < 8; u++) y[u] = src[(8 * j + u) * 512 + c];
    r8_inv(y, tw, 16 + j, 32 + 2 * j, 64 + 4 * j, q);
#pragma unroll
    for (int u = 0; u < 8; u++) sm[(8 * j + u) * kColTile + lane] = y[u];
  }
  __syncthreads();
  u64 x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = sm[(w + 8 * k) * kColTile + lane];
  r16_cols_inv(x, tw, q);
  const bool centre_out = (rd.flags & kCentre) != 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    u64 v = red2q(shoup(x[k], rd.c0, rd.c0s, q), q);
    if (centre_out) v = static_cast<u64>(centre(v, q));
    rd.dst[(w + 8 * k) * 512 + c] = v;
  }
}

// base conversion: a thread loads its coefficient's K sources once and
// produces every target; the table and the targets' primes sit in shared
// memory
__global__ void __launch_bounds__(256) k64_bconv(const __grid_constant__ BConv64Batch b) {
  __shared__ i64 tab[64 * 16];
  __shared__ u64 sp[64];
  __shared__ i64 sq[64];
  const BConv64Job &j = b.jobs[blockIdx.y];
  const int K = j.K, M = j.M;
  for (int t = threadIdx.x; t < M * K; t += blockDim.x) tab[t] = j.table[t];
  for (int t = threadIdx.x; t < M; t += blockDim.x) {
    sp[t] = b.primes[j.out_gidx[t]];
    sq[t] = b.qinvs[j.out_gidx[t]];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  i64 x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = k < K ? j.xt[(static_cast<size_t>(k) << 16) + i] : 0;
  for (int m = 0; m < M; m++) {
    const i64 *tm = tab + m * K;
    i128 acc = 0;
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k < K) acc += static_cast<i128>(x[k]) * tm[k];
    j.out[(static_cast<size_t>(j.out_row[m]) << 16) + i] = redc(acc, sp[m], sq[m]);
  }
}

__global__ void __launch_bounds__(256) k64_tensor(const __grid_constant__ Elem64Batch b) {
  const Elem64Row &e = b.rows[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const u64 b1 = e.b1[i], a1 = e.a1[i], b2 = e.b2[i], a2 = e.a2[i];
  e.o0[i] = mont_mul(b1, b2, e.q, e.qinv);
  e.o1[i] = add_mod(mont_mul(b1, a2, e.q, e.qinv), mont_mul(a1, b2, e.q, e.qinv), e.q);
  e.o2[i] = mont_mul(a1, a2, e.q, e.qinv);
}

__global__ void __launch_bounds__(256) k64_add(const __grid_constant__ Elem64Batch b) {
  const Elem64Row &e = b.rows[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  e.o0[i] = add_mod(e.a1[i], e.b1[i], e.q);
}

template <Elem64Op OP>
__global__ void __launch_bounds__(256) k64_elem(const __grid_constant__ Elem64Batch b) {
  const Elem64Row &e = b.rows[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const u64 q = e.q, x = e.a1[i];
  u64 o;
  switch (OP) {
    case Elem64Op::kAdd: o = add_mod(x, e.b1[i], q); break;
    case Elem64Op::kSub: o = red2q(x + q - e.b1[i], q); break;
    case Elem64Op::kNeg: o = x ? q - x : 0; break;
    case Elem64Op::kMult: o = mont_mul(x, e.b1[i], q, e.qinv); break;
    case Elem64Op::kMultConst: o = mont_mul(x, e.c, q, e.qinv); break;
    case Elem64Op::kAddConst: o = add_mod(x, e.c, q); break;
    case Elem64Op::kCopy: o = x; break;
    case Elem64Op::kMultImagUnit: o = mont_mul(x, (i & 32768) ? q - e.c : e.c, q, e.qinv); break;
  }
  e.o0[i] = o;
}

__device__ __forceinline__ uint32_t brev17(uint32_t x) { return __brev(x) >> 15; }

__global__ void __launch_bounds__(256) k64_permute(const __grid_constant__ Elem64Batch b, u64 galois) {
  const Elem64Row &e = b.rows[blockIdx.y];
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t ex = (brev17(k) + 1u) * static_cast<uint32_t>(galois) - 1u;
  const uint32_t src = brev17(ex & ((1u << 17) - 1u));
  e.o0[k] = e.a1[src];
}

__global__ void __launch_bounds__(256) k64_key_mac(const __grid_constant__ KeyMac64Batch b) {
  const KeyMac64Row &r = b.rows[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const u64 q = r.q;
  u64 sb = 0, sa = 0;
  for (int d = 0; d < r.beta; d++) {
    const u64 v = r.mu[d][i];
    sb = add_mod(sb, mont_mul(v, r.kb[d][i], q, r.qinv), q);
    sa = add_mod(sa, mont_mul(v, r.ka[d][i], q, r.qinv), q);
  }
  if (r.d0) sb = add_mod(sb, mont_mul(r.d0[i], r.p, q, r.qinv), q);
  if (r.d1) sa = add_mod(sa, mont_mul(r.d1[i], r.p, q, r.qinv), q);
  r.acc_b[i] = sb;
  r.acc_a[i] = sa;
}

}  // namespace

void launch_ntt64_fwd(const RowBatch64 &rb, cudaStream_t s) {
  if (rb.count <= 0) return;
  k64_fwd_cols<<<dim3(512 / kColTile, rb.count), 256, 0, s>>>(rb);
  k64_fwd_rows<<<dim3(128 / 4, rb.count), 256, 0, s>>>(rb);
}

void launch_ntt64_inv(const RowBatch64 &rb, cudaStream_t s) {
  if (rb.count <= 0) return;
  k64_inv_rows<<<dim3(128 / 4, rb.count), 256, 0, s>>>(rb);
  k64_inv_cols<<<dim3(512 / kColTile, rb.count), 256, 0, s>>>(rb);
}

void launch_bconv64(const BConv64Batch &b, cudaStream_t s) {
  if (b.count <= 0) return;
  k64_bconv<<<dim3(65536 / 256, b.count), 256, 0, s>>>(b);
}

void launch_tensor64(const Elem64Batch &b, cudaStream_t s) {
  if (b.count <= 0) return;
  k64_tensor<<<dim3(65536 / 256, b.count), 256, 0, s>>>(b);
}

void launch_add64(const Elem64Batch &b, cudaStream_t s) {
  if (b.count <= 0) return;
  k64_add<<<dim3(65536 / 256, b.count), 256, 0, s>>>(b);
}

void launch_elem64(Elem64Op op, const Elem64Batch &b, cudaStream_t s) {
  if (b.count <= 0) return;
  const dim3 grid(65536 / 256, b.count);
  switch (op) {
    case Elem64Op::kAdd: k64_elem<Elem64Op::kAdd><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kSub: k64_elem<Elem64Op::kSub><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kNeg: k64_elem<Elem64Op::kNeg><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kMult: k64_elem<Elem64Op::kMult><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kMultConst: k64_elem<Elem64Op::kMultConst><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kAddConst: k64_elem<Elem64Op::kAddConst><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kCopy: k64_elem<Elem64Op::kCopy><<<grid, 256, 0, s>>>(b); break;
    case Elem64Op::kMultImagUnit: k64_elem<Elem64Op::kMultImagUnit><<<grid, 256, 0, s>>>(b); break;
  }
}

void launch_permute64(const Elem64Batch &b, u64 galois, cudaStream_t s) {
  if (b.count <= 0) return;
  k64_permute<<<dim3(65536 / 256, b.count), 256, 0, s>>>(b, galois);
}

void launch_key_mac64(const KeyMac64Batch &b, cudaStream_t s) {
  if (b.count <= 0) return;
  k64_key_mac<<<dim3(65536 / 256, b.count), 256, 0, s>>>(b);
}

}  // namespace w64
}  // namespace chd
