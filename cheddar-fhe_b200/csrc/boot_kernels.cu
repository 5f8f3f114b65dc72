// Kernels of the bootstrapping path that the key-switching core does not have.
//
//  * k_modup_to_max: the exact lift of a level -1 polynomial (one or two base
//    primes, coefficient domain) to every prime of the top level
//    (kernel::ModUpToMax1 / ModUpToMax2, src/core/ElementWise.cu:575-623):
//    two base primes are combined by CRT into the centred representative
//    of (-q0 q1 / 2, q0 q1 / 2]; one base prime is lifted as is.
//  * k_pt_accum: sum_i pt_i (.) ct_i over limbs for several outputs and
//    several ciphertexts at once (the giant-step plaintext accumulation of
//    HoistHandler::GSFusedPAccum, src/extension/Hoist.cu:329-420, and
//    ElementWiseHandler::PAccum).
//  * k_const_accum: sum_i c_i * ct_i with one constant per limb and term
//    (ElementWiseHandler::CAccum, src/core/ElementWise.cu:1355-1643).
#include "arith.cuh"
#include "kernels.h"

namespace chd {
namespace {

__global__ void k_modup_to_max(const __grid_constant__ ModUpToMaxDesc d) {
  const int r = blockIdx.y;
  const int part = blockIdx.z;
  const uint32_t p = d.p[r];
  const size_t n = static_cast<size_t>(d.n);
  const uint32_t *src = d.src[part];
  uint32_t *dst = d.dst[part] + static_cast<size_t>(r) * n;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    if (d.nbase == 1) {
      dst[i] = src[i] % p;
    } else {
      const int64_t q0 = d.q0, q1 = d.q1;
      const int64_t qp = q0 * q1;
      int64_t v = static_cast<int64_t>(src[i]) * q1 + static_cast<int64_t>(src[n + i]) * q0;
      if (v >= qp) v -= qp;
      if (v > (qp >> 1)) v -= qp;
      int64_t m = v % static_cast<int64_t>(p);
      if (m < 0) m += p;
      dst[i] = static_cast<uint32_t>(m);
    }
  }
}

// out[c][o][r] = sum_t pt[o][t][r] (.) in[c][t][r]  (Montgomery products,
// canonical).  One thread owns one coefficient of one row of one ciphertext:
// it reads each baby-step value once and keeps the G giant-step sums in
// registers, so no value is re-read.  Block x = ciphertext + count * column
// block: the blocks of a batch that read the same plaintext tile run back to
// back and share it through L2.
template <int G>
__global__ void __launch_bounds__(256) k_pt_accum(const __grid_constant__ PtAccumDesc d) {
  const int r = blockIdx.y;
  const int c = blockIdx.x % d.count, xb = blockIdx.x / d.count;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t i = static_cast<size_t>(xb) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(d.n)) return;
  const size_t idx = static_cast<size_t>(r) * d.n + i;
  uint32_t sb[G], sa[G];
#pragma unroll
  for (int o = 0; o < G; o++) sb[o] = sa[o] = 0;
  for (int t = 0; t < d.ins; t++) {
    const uint32_t xb_ = d.in_b[c][t][idx], xa_ = d.in_a[c][t][idx];
#pragma unroll
    for (int o = 0; o < G; o++) {
      const uint32_t *p = d.pt[o][t];
      if (o < d.outs && p != nullptr) {
        const uint32_t m = p[idx];
        sb[o] = add_mod(sb[o], mont_mul(xb_, m, q, qi), q);
        sa[o] = add_mod(sa[o], mont_mul(xa_, m, q, qi), q);
      }
    }
  }
#pragma unroll
  for (int o = 0; o < G; o++)
    if (o < d.outs) {
      d.out_b[c][o][idx] = sb[o];
      d.out_a[c][o][idx] = sa[o];
    }
}

// dst[p][r] = sum_t c[t][r] * src[t][p][r]  (Montgomery constants, canonical)
__global__ void k_const_accum(const __grid_constant__ ConstAccumDesc d) {
  const int r = blockIdx.y;
  const int part = blockIdx.z;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t n = static_cast<size_t>(d.n);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint32_t s = 0;
    for (int t = 0; t < d.terms; t++) {
      const uint32_t *src = d.src[t][part] + static_cast<size_t>(d.src_row0[t] + r) * n;
      s = add_mod(s, mont_mul(src[i], d.c[t][r], q, qi), q);
    }
    d.dst[part][static_cast<size_t>(r) * n + i] = s;
  }
}

}  // namespace

void launch_modup_to_max(const ModUpToMaxDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.parts <= 0) return;
  k_modup_to_max<<<dim3(64, d.rows, d.parts), 256, 0, s>>>(d);
}

void launch_pt_accum(const PtAccumDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.rows > 64 || d.outs <= 0 || d.outs > kMaxPtAccumOuts || d.ins <= 0 ||
      d.ins > kMaxPtAccumIn || d.count <= 0 || d.count > kMaxPtAccumCts)
    return;
  const dim3 grid(d.count * ((d.n + 255) / 256), d.rows);
  if (d.outs <= 1)
    k_pt_accum<1><<<grid, 256, 0, s>>>(d);
  else if (d.outs <= 4)
    k_pt_accum<4><<<grid, 256, 0, s>>>(d);
  else if (d.outs <= 8)
    k_pt_accum<8><<<grid, 256, 0, s>>>(d);
  else
    k_pt_accum<16><<<grid, 256, 0, s>>>(d);
}

void launch_const_accum(const ConstAccumDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.parts <= 0 || d.terms <= 0) return;
  k_const_accum<<<dim3(64, d.rows, d.parts), 256, 0, s>>>(d);
}

}  // namespace chd
