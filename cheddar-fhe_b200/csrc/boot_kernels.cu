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
// canonical).  Block x = ciphertext + count * column block: the blocks of the
// ciphertexts of one batch that read the same plaintext tile are neighbours
// in launch order, so the plaintexts come from HBM once per batch.  One
// thread owns one coefficient of one row for every output, so the baby-step
// values it reads for the first giant step are L1 hits for the others.
__global__ void k_pt_accum(const __grid_constant__ PtAccumDesc d) {
  const int r = blockIdx.y;
  const int c = blockIdx.x % d.count, xb = blockIdx.x / d.count, nxb = gridDim.x / d.count;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t n = static_cast<size_t>(d.n);
  const size_t off = static_cast<size_t>(r) * n;
  for (size_t i = xb * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(nxb) * blockDim.x) {
    for (int o = 0; o < d.outs; o++) {
      const PtAccumOut &out = d.out[o];
      uint32_t sb = 0, sa = 0;
      for (int t = 0; t < out.terms; t++) {
        const int ti = out.term[t];
        const uint32_t m = out.pt[t][off + i];
        sb = add_mod(sb, mont_mul(d.in_b[c][ti][off + i], m, q, qi), q);
        sa = add_mod(sa, mont_mul(d.in_a[c][ti][off + i], m, q, qi), q);
      }
      d.out_b[c][o][off + i] = sb;
      d.out_a[c][o][off + i] = sa;
    }
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
  if (d.rows <= 0 || d.outs <= 0 || d.count <= 0 || d.count > kMaxPtAccumCts) return;
  k_pt_accum<<<dim3(64 * d.count, d.rows), 256, 0, s>>>(d);
}

void launch_const_accum(const ConstAccumDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.parts <= 0 || d.terms <= 0) return;
  k_const_accum<<<dim3(64, d.rows, d.parts), 256, 0, s>>>(d);
}

}  // namespace chd
