// Building blocks shared by the NTT kernels (ntt.cu), the fused ModSwitch
// column pass (modswitch.cu) and the fused key-switch row pass
// (keyswitch.cu): radix-8 / radix-16 networks of lazy Shoup butterflies with
// vectorised twiddle loads, and the shared-memory swizzle of the row phase.
#pragma once

#include "arith.cuh"

namespace chd {

// Twiddle loads: tables hold (w, companion) pairs; pairs at even (resp.
// multiple-of-4) indices are 16- (resp. 32-) byte aligned, so 2 and 4
// consecutive pairs are fetched with 128-bit loads.
__device__ __forceinline__ void tw_ld2(const uint2 *tw, int i, uint2 *w) {
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(tw + i));
  w[0] = make_uint2(v.x, v.y);
  w[1] = make_uint2(v.z, v.w);
}
__device__ __forceinline__ void tw_ld4(const uint2 *tw, int i, uint2 *w) {
  tw_ld2(tw, i, w);
  tw_ld2(tw, i + 2, w + 2);
}

// Radix-8 forward network on x[0..7]: CT stages at register distances 4, 2,
// 1 with twiddles tw[b0], tw[b1 + g] (g < 2), tw[b2 + g] (g < 4).
// b1 must be even and b2 a multiple of 4.
__device__ __forceinline__ void radix8_fwd(uint32_t *x, const uint2 *tw, int b0, int b1, int b2, uint32_t q) {
  uint2 w1[2], w2[4];
  const uint2 w0 = __ldg(tw + b0);
  tw_ld2(tw, b1, w1);
  tw_ld4(tw, b2, w2);
#pragma unroll
  for (int k = 0; k < 4; k++) ct_lazy(x[k], x[k + 4], w0, q);
#pragma unroll
  for (int g = 0; g < 2; g++) {
    ct_lazy(x[4 * g], x[4 * g + 2], w1[g], q);
    ct_lazy(x[4 * g + 1], x[4 * g + 3], w1[g], q);
  }
#pragma unroll
  for (int g = 0; g < 4; g++) ct_lazy(x[2 * g], x[2 * g + 1], w2[g], q);
}

// Radix-8 inverse network (GS stages at distances 1, 2, 4), mirror of the above.
__device__ __forceinline__ void radix8_inv(uint32_t *x, const uint2 *tw, int b0, int b1, int b2, uint32_t q) {
  uint2 w1[2], w2[4];
  const uint2 w0 = __ldg(tw + b0);
  tw_ld2(tw, b1, w1);
  tw_ld4(tw, b2, w2);
#pragma unroll
  for (int g = 0; g < 4; g++) gs_lazy(x[2 * g], x[2 * g + 1], w2[g], q);
#pragma unroll
  for (int g = 0; g < 2; g++) {
    gs_lazy(x[4 * g], x[4 * g + 2], w1[g], q);
    gs_lazy(x[4 * g + 1], x[4 * g + 3], w1[g], q);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) gs_lazy(x[k], x[k + 4], w0, q);
}

// First four column stages (m = 1, 2, 4, 8) on 16 registers holding rows
// rg + 8k of one column: pair (k, k + 8/m) with twiddle tw[m + k / (16/m)].
__device__ __forceinline__ void radix16_cols_fwd(uint32_t *x, const uint2 *tw, uint32_t q) {
  uint2 w[16];
  w[1] = __ldg(tw + 1);
  tw_ld2(tw, 2, w + 2);
  tw_ld4(tw, 4, w + 4);
  tw_ld4(tw, 8, w + 8);
  tw_ld4(tw, 12, w + 12);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int m = 1 << s, h = 8 >> s;
#pragma unroll
    for (int g = 0; g < m; g++)
#pragma unroll
      for (int j = 0; j < h; j++) ct_lazy(x[g * 2 * h + j], x[g * 2 * h + j + h], w[m + g], q);
  }
}

// Last four inverse column stages (m = 8, 4, 2, 1), mirror of the above.
__device__ __forceinline__ void radix16_cols_inv(uint32_t *x, const uint2 *tw, uint32_t q) {
  uint2 w[16];
  w[1] = __ldg(tw + 1);
  tw_ld2(tw, 2, w + 2);
  tw_ld4(tw, 4, w + 4);
  tw_ld4(tw, 8, w + 8);
  tw_ld4(tw, 12, w + 12);
#pragma unroll
  for (int s = 3; s >= 0; s--) {
    const int m = 1 << s, h = 8 >> s;
#pragma unroll
    for (int g = 0; g < m; g++)
#pragma unroll
      for (int j = 0; j < h; j++) gs_lazy(x[g * 2 * h + j], x[g * 2 * h + j + h], w[m + g], q);
  }
}

// Shared-memory position of element c of a 512-element row.  The three
// exchange patterns of the row phase (c = t + 64k, 64(t>>3) + (t&7) + 8k and
// 8t + k, t the lane) are all bank-conflict free under this bijection.
__device__ __forceinline__ int rsw(int c) { return c ^ ((c >> 3) & 31); }

// Barrier of the 64 threads (two warps) that own one row: named barrier
// `bar` (1 .. 15), so that the rows of a CTA do not wait for each other, or
// the CTA-wide barrier for bar < 0.  The key-switch row pass (several loads
// and MACs between its row transforms) gains from the per-row form; the
// plain row kernels measured faster with the CTA-wide one.
__device__ __forceinline__ void row_sync(int bar) {
  if (bar < 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory");
}

// The 9 row stages (m = 128 .. 32768) of the forward transform on one
// 512-element row r held by 64 threads (thread t), 8 elements each.  Input
// x[k] = element t + 64k; output x[k] = element 8t + k.  srow is the row's
// 512-word shared buffer, bar the row's named barrier; the caller
// synchronises (row_sync) before reusing srow.
__device__ __forceinline__ void row_fwd(uint32_t *x, uint32_t *srow, const uint2 *tw, int r, int t, uint32_t q,
                                        int bar) {
  const int b = t >> 3, u0 = t & 7;
  radix8_fwd(x, tw, 128 + r, 256 + 2 * r, 512 + 4 * r, q);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(t + 64 * k)] = x[k];
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(64 * b + u0 + 8 * k)];
  radix8_fwd(x, tw, 1024 + 8 * r + b, 2048 + 16 * r + 2 * b, 4096 + 32 * r + 4 * b, q);
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(64 * b + u0 + 8 * k)] = x[k];
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(8 * t + k)];
  radix8_fwd(x, tw, 8192 + 64 * r + t, 16384 + 128 * r + 2 * t, 32768 + 256 * r + 4 * t, q);
}

// The 9 row stages of the inverse transform (m = 32768 .. 128): input x[k] =
// element 8t + k, output x[k] = element t + 64k.
__device__ __forceinline__ void row_inv(uint32_t *x, uint32_t *srow, const uint2 *tw, int r, int t, uint32_t q,
                                        int bar) {
  const int b = t >> 3, u0 = t & 7;
  radix8_inv(x, tw, 8192 + 64 * r + t, 16384 + 128 * r + 2 * t, 32768 + 256 * r + 4 * t, q);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(8 * t + k)] = x[k];
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(64 * b + u0 + 8 * k)];
  radix8_inv(x, tw, 1024 + 8 * r + b, 2048 + 16 * r + 2 * b, 4096 + 32 * r + 4 * b, q);
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) srow[rsw(64 * b + u0 + 8 * k)] = x[k];
  row_sync(bar);
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = srow[rsw(t + 64 * k)];
  radix8_inv(x, tw, 128 + r, 256 + 2 * r, 512 + 4 * r, q);
}

__device__ __forceinline__ void ld8(const uint32_t *p, uint32_t *x) {
  const uint4 *v = reinterpret_cast<const uint4 *>(p);
  const uint4 a = __ldg(v), b = __ldg(v + 1);
  x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
  x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}
__device__ __forceinline__ void st8(uint32_t *p, const uint32_t *x) {
  uint4 *v = reinterpret_cast<uint4 *>(p);
  v[0] = make_uint4(x[0], x[1], x[2], x[3]);
  v[1] = make_uint4(x[4], x[5], x[6], x[7]);
}

}  // namespace chd
