// Base conversion, key-switching inner product, element-wise and
// automorphism kernels.  All are HBM-streaming integer kernels: each thread
// owns 4 consecutive coefficients (128-bit loads and stores), grid.y walks
// the limbs (or jobs) of the batch.
#include <map>
#include <mutex>
#include <tuple>

#include "arith.cuh"
#include "kernels.h"

namespace chd {
namespace {

__device__ __forceinline__ uint4 ld4(const uint32_t *p) { return __ldg(reinterpret_cast<const uint4 *>(p)); }
__device__ __forceinline__ void st4(uint32_t *p, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  *reinterpret_cast<uint4 *>(p) = make_uint4(a, b, c, d);
}
__device__ __forceinline__ void unpack(uint4 v, uint32_t *x) {
  x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
}

// ------------------------------------------------------------------ BConv
// out[m][n] = (sum_k xt[k][n] T[m][k]) * 2^-32 mod p_m, exact.  |xt| < 2^30
// and |T| <= (p-1)/2 bound every product by p * 2^29, so a group of 4 terms
// stays inside the (-p 2^31, p 2^31) input range of the Montgomery reduction;
// group results are summed canonically.  (The reference kernel,
// src/core/ModSwitch.cu:23-171, computes the same residue.)
constexpr int kBConvTargetsPerCta = 8;

template <int KMAX>
__global__ void __launch_bounds__(256) k_bconv(const __grid_constant__ BConvBatch b, int log_n) {
  const BConvJob &jb = b.jobs[blockIdx.y];
  const int m0 = blockIdx.z * kBConvTargetsPerCta;
  if (m0 >= jb.M) return;
  const int m1 = min(m0 + kBConvTargetsPerCta, jb.M);
  const int n = 1 << log_n;
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 2;
  if (i0 >= n) return;
  const int K = jb.K;
  int32_t x[KMAX][2];
#pragma unroll
  for (int k = 0; k < KMAX; k++) {
    if (k < K) {
      int2 v = __ldg(reinterpret_cast<const int2 *>(jb.xt + static_cast<size_t>(k) * n + i0));
      x[k][0] = v.x;
      x[k][1] = v.y;
    }
  }
  for (int m = m0; m < m1; m++) {
    const int g = jb.out_gidx[m];
    const uint32_t p = __ldg(b.primes + g);
    const int32_t pinv = __ldg(b.qinvs + g);
    const int32_t *T = jb.table + m * K;
    uint32_t s0 = 0, s1 = 0;
#pragma unroll
    for (int k0 = 0; k0 < KMAX; k0 += 4) {
      if (k0 < K) {
        int64_t a0 = 0, a1 = 0;
#pragma unroll
        for (int k = k0; k < k0 + 4; k++) {
          if (k < K) {
            const int64_t t = __ldg(T + k);
            a0 += static_cast<int64_t>(x[k][0]) * t;
            a1 += static_cast<int64_t>(x[k][1]) * t;
          }
        }
        s0 = add_mod(s0, mont_reduce(a0, p, pinv), p);
        s1 = add_mod(s1, mont_reduce(a1, p, pinv), p);
      }
    }
    *reinterpret_cast<uint2 *>(jb.out + static_cast<size_t>(jb.out_row[m]) * n + i0) = make_uint2(s0, s1);
  }
}

// ---------------------------------------------------------------- key MAC
__global__ void __launch_bounds__(256) k_key_mac(const __grid_constant__ KeyMacDesc d, int log_n) {
  const int n = 1 << log_n;
  // block x = ciphertext + count * column block: the ciphertexts reading
  // the same key tile are neighbours in launch order (the key comes from HBM
  // once per batch)
  const int r = blockIdx.y;
  const KeyMacCt &c = d.ct[blockIdx.x % d.count];
  const int i0 = ((blockIdx.x / d.count) * blockDim.x + threadIdx.x) * 4;
  if (i0 >= n) return;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t off = static_cast<size_t>(r) * n + i0;
  const size_t koff = static_cast<size_t>(d.key_row[r]) * n + i0;
  const uint32_t qn = 0u - static_cast<uint32_t>(qi);
  uint32_t sb[4] = {0, 0, 0, 0}, sa[4] = {0, 0, 0, 0};
  int i = 0;
  for (; i + 1 < d.beta; i += 2) {  // two digits per Montgomery reduction
    uint32_t mu0[4], kb0[4], ka0[4], mu1[4], kb1[4], ka1[4];
    unpack(ld4(c.mu[i] + off), mu0);
    unpack(ld4(d.kb[i] + koff), kb0);
    unpack(ld4(d.ka[i] + koff), ka0);
    unpack(ld4(c.mu[i + 1] + off), mu1);
    unpack(ld4(d.kb[i + 1] + koff), kb1);
    unpack(ld4(d.ka[i + 1] + koff), ka1);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      sb[l] = add_mod(sb[l], mont_mac2(mu0[l], kb0[l], mu1[l], kb1[l], q, qn), q);
      sa[l] = add_mod(sa[l], mont_mac2(mu0[l], ka0[l], mu1[l], ka1[l], q, qn), q);
    }
  }
  if (i < d.beta) {
    uint32_t mu[4], kb[4], ka[4];
    unpack(ld4(c.mu[i] + off), mu);
    unpack(ld4(d.kb[i] + koff), kb);
    unpack(ld4(d.ka[i] + koff), ka);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      sb[l] = add_mod(sb[l], mont_mul(mu[l], kb[l], q, qi), q);
      sa[l] = add_mod(sa[l], mont_mul(mu[l], ka[l], q, qi), q);
    }
  }
  if (r < d.nq) {
    const uint32_t pp = d.p_prod[r];
    if (c.d0) {
      uint32_t v[4];
      unpack(ld4(c.d0 + off), v);
#pragma unroll
      for (int l = 0; l < 4; l++) sb[l] = add_mod(sb[l], mont_mul(v[l], pp, q, qi), q);
    }
    if (c.d1) {
      uint32_t v[4];
      unpack(ld4(c.d1 + off), v);
#pragma unroll
      for (int l = 0; l < 4; l++) sa[l] = add_mod(sa[l], mont_mul(v[l], pp, q, qi), q);
    }
  }
  st4(c.acc_b + off, sb[0], sb[1], sb[2], sb[3]);
  st4(c.acc_a + off, sa[0], sa[1], sa[2], sa[3]);
}

// ----------------------------------------------------------- element-wise
template <ElemOp OP>
__global__ void __launch_bounds__(256) k_elem(const __grid_constant__ ElemBatch eb, int log_n) {
  const int n = 1 << log_n;
  const ElemRow &e = eb.rows[blockIdx.y];
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i0 >= n) return;
  const uint32_t q = e.q;
  const int32_t qi = e.qinv;
  uint32_t a[4], b[4], c[4], o[4];
  unpack(ld4(e.a + i0), a);
  if (OP == ElemOp::kAdd || OP == ElemOp::kSub || OP == ElemOp::kMult || OP == ElemOp::kMultAdd)
    unpack(ld4(e.b + i0), b);
  if (OP == ElemOp::kMultAdd || OP == ElemOp::kMultConstAdd) unpack(ld4(e.c + i0), c);
#pragma unroll
  for (int l = 0; l < 4; l++) {
    switch (OP) {
      case ElemOp::kAdd: o[l] = add_mod(a[l], b[l], q); break;
      case ElemOp::kSub: o[l] = sub_mod(a[l], b[l], q); break;
      case ElemOp::kNeg: o[l] = neg_mod(a[l], q); break;
      case ElemOp::kMult: o[l] = mont_mul(a[l], b[l], q, qi); break;
      case ElemOp::kAddConst: o[l] = add_mod(a[l], e.k, q); break;
      case ElemOp::kSubConst: o[l] = sub_mod(a[l], e.k, q); break;
      case ElemOp::kSubOppConst: o[l] = sub_mod(e.k, a[l], q); break;
      case ElemOp::kMultConst: o[l] = mont_mul(a[l], e.k, q, qi); break;
      case ElemOp::kCopy: o[l] = a[l]; break;
      case ElemOp::kMultImagUnit: {
        // X^(N/2) in the bit-reversed evaluation domain: +-psi^(N/2)
        const uint32_t u = ((i0 + l) & (n >> 1)) ? q - e.k : e.k;
        o[l] = mont_mul(a[l], u, q, qi);
        break;
      }
      case ElemOp::kMultAdd: o[l] = add_mod(c[l], mont_mul(a[l], b[l], q, qi), q); break;
      case ElemOp::kMultConstAdd: o[l] = add_mod(c[l], mont_mul(a[l], e.k, q, qi), q); break;
    }
  }
  st4(e.dst + i0, o[0], o[1], o[2], o[3]);
}

__global__ void __launch_bounds__(256) k_tensor(const __grid_constant__ TensorBatch tb, int log_n) {
  const int n = 1 << log_n;
  const TensorRow &t = tb.rows[blockIdx.y];
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i0 >= n) return;
  const uint32_t q = t.q;
  const int32_t qi = t.qinv;
  uint32_t b1[4], a1[4], b2[4], a2[4], o0[4], o1[4], o2[4];
  unpack(ld4(t.b1 + i0), b1);
  unpack(ld4(t.a1 + i0), a1);
  unpack(ld4(t.b2 + i0), b2);
  unpack(ld4(t.a2 + i0), a2);
#pragma unroll
  for (int l = 0; l < 4; l++) {
    o0[l] = mont_mul(b1[l], b2[l], q, qi);
    o2[l] = mont_mul(a1[l], a2[l], q, qi);
    o1[l] = mont_mac2(b1[l], a2[l], a1[l], b2[l], q, 0u - static_cast<uint32_t>(qi));
  }
  st4(t.d0 + i0, o0[0], o0[1], o0[2], o0[3]);
  st4(t.d1 + i0, o1[0], o1[1], o1[2], o1[3]);
  st4(t.d2 + i0, o2[0], o2[1], o2[2], o2[3]);
}

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int bits) { return __brev(x) >> (32 - bits); }

// source index of the automorphism gather for destination k
__device__ __forceinline__ uint32_t galois_src(uint32_t k, uint32_t g, int log_n) {
  const int lb = log_n + 1;
  const uint32_t e = (brev_bits(k, lb) + 1u) * g - 1u;
  return brev_bits(e & ((1u << lb) - 1u), lb);
}

// dst[k] = src[galois_src(k)] (+ add[k]).  An aligned group of 4
// destinations gathers from one aligned group of 4 sources (the bit-reversed
// automorphism only reorders the two low bits), so every thread moves 4
// coefficients with one 16-byte load and store each.
__global__ void __launch_bounds__(256) k_permute(const __grid_constant__ PermuteBatch pb, int log_n) {
  const int n = 1 << log_n;
  const PermuteRow &p = pb.rows[blockIdx.y];
  const int k0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (k0 >= n) return;
  uint32_t slot[4];
#pragma unroll
  for (int l = 0; l < 4; l++) slot[l] = galois_src(k0 + l, pb.galois, log_n);
  uint32_t x[4], v[4];
  unpack(ld4(p.src + (slot[0] & ~3u)), x);
  if (p.src2) {
    uint32_t y[4];
    unpack(ld4(p.src2 + (slot[0] & ~3u)), y);
#pragma unroll
    for (int l = 0; l < 4; l++) x[l] = add_mod(x[l], y[l], p.q);
  }
#pragma unroll
  for (int l = 0; l < 4; l++) {
    const uint32_t m = slot[l] & 3u;
    v[l] = m == 0 ? x[0] : m == 1 ? x[1] : m == 2 ? x[2] : x[3];
  }
  if (p.add) {
    uint32_t a[4];
    unpack(ld4(p.add + k0), a);
#pragma unroll
    for (int l = 0; l < 4; l++) v[l] = add_mod(v[l], a[l], p.q);
  }
  st4(p.dst + k0, v[0], v[1], v[2], v[3]);
}

// Hoisted rotations (one launch for all R rotations).  Each thread loads the
// beta ModUp values of 4 adjacent coefficients once, then for every rotation
// forms the key inner products and stores them through the inverse
// automorphism.  In the bit-reversed domain the automorphism maps an aligned
// group of 4 coefficients onto an aligned group of 4 (only the two top bits
// of the exponent differ, and they become the two low bits of the
// destination), so the 4 results leave as one 16-byte store after a
// permutation in registers.  Grid (count, N / 1024, rows): the ciphertexts of
// a batch that read the same key tile are neighbours in launch order, so the
// keys come from HBM once per batch.
// BMAX: digits held per thread; with at most 4 (every parameter set here at
// the levels hoisted rotations run at) the kernel fits 3 CTAs per SM (MINB)
// instead of 2, or 4 with a few words spilled
template <int BMAX, int MINB>
__global__ void __launch_bounds__(256, MINB) k_hoisted(const __grid_constant__ HoistDesc d, int log_n) {
  const int n = 1 << log_n;
  const int c = blockIdx.x;
  const int r = blockIdx.z;
  const int k0 = (blockIdx.y * blockDim.x + threadIdx.x) * 4;
  if (k0 >= n) return;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t off = static_cast<size_t>(r) * n + k0;
  const size_t koff = static_cast<size_t>(d.key_row[r]) * n + k0;
  const uint32_t qn = 0u - static_cast<uint32_t>(qi);
  uint32_t mu[BMAX][4];
#pragma unroll
  for (int i = 0; i < BMAX; i++)
    if (i < d.beta) unpack(ld4(d.mu[c][i] + off), mu[i]);
  uint32_t bxp[4] = {0, 0, 0, 0};
  if (r < d.nq) unpack(ld4(d.bxp[c] + off), bxp);
  for (int j = 0; j < d.R; j++) {
    uint32_t sb[4], sa[4] = {0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < 4; l++) sb[l] = bxp[l];
#pragma unroll
    for (int i = 0; i < BMAX; i += 2) {
      if (i + 1 < d.beta) {  // two digits per Montgomery reduction
        uint32_t kb0[4], ka0[4], kb1[4], ka1[4];
        unpack(ld4(d.kb[j][i] + koff), kb0);
        unpack(ld4(d.ka[j][i] + koff), ka0);
        unpack(ld4(d.kb[j][i + 1] + koff), kb1);
        unpack(ld4(d.ka[j][i + 1] + koff), ka1);
#pragma unroll
        for (int l = 0; l < 4; l++) {
          sb[l] = add_mod(sb[l], mont_mac2(mu[i][l], kb0[l], mu[i + 1][l], kb1[l], q, qn), q);
          sa[l] = add_mod(sa[l], mont_mac2(mu[i][l], ka0[l], mu[i + 1][l], ka1[l], q, qn), q);
        }
      } else if (i < d.beta) {
        uint32_t kb[4], ka[4];
        unpack(ld4(d.kb[j][i] + koff), kb);
        unpack(ld4(d.ka[j][i] + koff), ka);
#pragma unroll
        for (int l = 0; l < 4; l++) {
          sb[l] = add_mod(sb[l], mont_mul(mu[i][l], kb[l], q, qi), q);
          sa[l] = add_mod(sa[l], mont_mul(mu[i][l], ka[l], q, qi), q);
        }
      }
    }
    uint32_t slot[4];
#pragma unroll
    for (int l = 0; l < 4; l++) slot[l] = galois_src(k0 + l, d.galois_inv[j], log_n);
    const size_t o = static_cast<size_t>(r) * n + (slot[0] & ~3u);
    uint32_t ob[4], oa[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const uint32_t u = static_cast<uint32_t>(m);
      ob[m] = (slot[0] & 3u) == u ? sb[0] : (slot[1] & 3u) == u ? sb[1] : (slot[2] & 3u) == u ? sb[2] : sb[3];
      oa[m] = (slot[0] & 3u) == u ? sa[0] : (slot[1] & 3u) == u ? sa[1] : (slot[2] & 3u) == u ? sa[2] : sa[3];
    }
    st4(d.out_b[c][j] + o, ob[0], ob[1], ob[2], ob[3]);
    st4(d.out_a[c][j] + o, oa[0], oa[1], oa[2], oa[3]);
  }
}

}  // namespace

void launch_bconv(const BConvBatch &b, int log_n, cudaStream_t s) {
  if (b.count <= 0) return;
  const int n = 1 << log_n;
  int max_m = 0;
  for (int j = 0; j < b.count; j++) max_m = b.jobs[j].M > max_m ? b.jobs[j].M : max_m;
  int max_k = 0;
  for (int j = 0; j < b.count; j++) max_k = b.jobs[j].K > max_k ? b.jobs[j].K : max_k;
  const int zs = (max_m + kBConvTargetsPerCta - 1) / kBConvTargetsPerCta;
  const dim3 grid((n / 2 + 255) / 256, b.count, zs);
  if (max_k <= 4)
    k_bconv<4><<<grid, 256, 0, s>>>(b, log_n);
  else if (max_k <= 8)
    k_bconv<8><<<grid, 256, 0, s>>>(b, log_n);
  else if (max_k <= 12)
    k_bconv<12><<<grid, 256, 0, s>>>(b, log_n);
  else
    k_bconv<16><<<grid, 256, 0, s>>>(b, log_n);
}

void launch_key_mac(const KeyMacDesc &d, int log_n, cudaStream_t s) {
  if (d.rows <= 0 || d.count <= 0) return;
  const int n = 1 << log_n;
  k_key_mac<<<dim3(d.count * ((n / 4 + 255) / 256), d.rows), 256, 0, s>>>(d, log_n);
}

void launch_elementwise(ElemOp op, const ElemBatch &b, int log_n, cudaStream_t s) {
  if (b.count <= 0) return;
  const int n = 1 << log_n;
  dim3 grid((n / 4 + 255) / 256, b.count);
  switch (op) {
#define CHD_CASE(OP) \
  case OP: k_elem<OP><<<grid, 256, 0, s>>>(b, log_n); break;
    CHD_CASE(ElemOp::kAdd)
    CHD_CASE(ElemOp::kSub)
    CHD_CASE(ElemOp::kNeg)
    CHD_CASE(ElemOp::kMult)
    CHD_CASE(ElemOp::kAddConst)
    CHD_CASE(ElemOp::kSubConst)
    CHD_CASE(ElemOp::kSubOppConst)
    CHD_CASE(ElemOp::kMultConst)
    CHD_CASE(ElemOp::kCopy)
    CHD_CASE(ElemOp::kMultImagUnit)
    CHD_CASE(ElemOp::kMultAdd)
    CHD_CASE(ElemOp::kMultConstAdd)
#undef CHD_CASE
  }
}

void launch_tensor(const TensorBatch &b, int log_n, cudaStream_t s) {
  if (b.count <= 0) return;
  const int n = 1 << log_n;
  k_tensor<<<dim3((n / 4 + 255) / 256, b.count), 256, 0, s>>>(b, log_n);
}

void launch_permute(const PermuteBatch &b, int log_n, cudaStream_t s) {
  if (b.count <= 0) return;
  const int n = 1 << log_n;
  k_permute<<<dim3((n / 4 + 255) / 256, b.count), 256, 0, s>>>(b, log_n);
}

namespace {
// Autotuning of the baby-step kernel (with CHD_BCONV_AUTO): for up to 4
// digits, the first launch of a shape (device, ciphertexts, rotations, rows,
// digits) outside a stream capture times the 3- and 4-CTA forms three times,
// interleaved, after a warm-up, and caches the faster; every launch writes
// the same words.
std::mutex g_hoist_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_hoist_cache;

void launch_hoisted_variant(const HoistDesc &d, int log_n, int variant, cudaStream_t s) {
  const int n = 1 << log_n;
  const dim3 grid(d.count, (n / 4 + 255) / 256, d.rows);
  if (d.beta > 4)
    k_hoisted<8, 2><<<grid, 256, 0, s>>>(d, log_n);
  else if (variant == 1)
    k_hoisted<4, 4><<<grid, 256, 0, s>>>(d, log_n);
  else
    k_hoisted<4, 3><<<grid, 256, 0, s>>>(d, log_n);
}
}  // namespace

void launch_hoisted(const HoistDesc &d, int log_n, cudaStream_t s, bool tune) {
  if (d.rows <= 0 || d.R <= 0) return;
  if (d.count <= 0 || d.count > kMaxHoistCts) return;
  if (!tune || d.beta > 4) {
    launch_hoisted_variant(d, log_n, 0, s);
    return;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, d.count, d.R, d.rows, d.beta);
  {
    std::lock_guard<std::mutex> lock(g_hoist_mu);
    auto it = g_hoist_cache.find(key);
    if (it != g_hoist_cache.end()) {
      launch_hoisted_variant(d, log_n, it->second, s);
      return;
    }
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    launch_hoisted_variant(d, log_n, 0, s);
    return;
  }
  constexpr int kVariants = 2, kReps = 3;
  cudaEvent_t ev[kVariants * kReps + 1] = {};
  for (auto &e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      for (auto &f : ev)
        if (f) cudaEventDestroy(f);
      launch_hoisted_variant(d, log_n, 0, s);
      return;
    }
  for (int v = 0; v < kVariants; v++) launch_hoisted_variant(d, log_n, v, s);
  cudaEventRecord(ev[0], s);
  for (int r = 0; r < kReps; r++)
    for (int v = 0; v < kVariants; v++) {
      launch_hoisted_variant(d, log_n, v, s);
      cudaEventRecord(ev[r * kVariants + v + 1], s);
    }
  bool ok = cudaEventSynchronize(ev[kVariants * kReps]) == cudaSuccess;
  float best[kVariants] = {1e30f, 1e30f};
  for (int r = 0; ok && r < kReps; r++)
    for (int v = 0; ok && v < kVariants; v++) {
      float t = 0.f;
      const int i = r * kVariants + v;
      ok = cudaEventElapsedTime(&t, ev[i], ev[i + 1]) == cudaSuccess;
      best[v] = t < best[v] ? t : best[v];
    }
  for (auto &e : ev) cudaEventDestroy(e);
  if (ok) {
    std::lock_guard<std::mutex> lock(g_hoist_mu);
    g_hoist_cache[key] = best[1] < best[0] ? 1 : 0;
  }
}

}  // namespace chd
