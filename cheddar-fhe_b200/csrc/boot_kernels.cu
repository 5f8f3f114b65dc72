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
#include <map>
#include <mutex>
#include <tuple>

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

template <int V>
__device__ __forceinline__ void ld_vec(const uint32_t *p, uint32_t (&x)[V]) {
  if constexpr (V == 4) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w;
  } else if constexpr (V == 2) {
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    x[0] = u.x, x[1] = u.y;
  } else {
    x[0] = *p;
  }
}
template <int V>
__device__ __forceinline__ void st_vec(uint32_t *p, const uint32_t (&x)[V]) {
  if constexpr (V == 4) {
    *reinterpret_cast<uint4 *>(p) = make_uint4(x[0], x[1], x[2], x[3]);
  } else if constexpr (V == 2) {
    *reinterpret_cast<uint2 *>(p) = make_uint2(x[0], x[1]);
  } else {
    *p = x[0];
  }
}

// out[c][o][r] = sum_t pt[o][t][r] (.) in[c][t][r]  (Montgomery products,
// canonical).  One thread owns V adjacent coefficients of one row of one
// ciphertext: it reads each baby-step value once (V-word vector loads) and
// keeps the G giant-step sums in registers, so no value is re-read; two baby
// steps share one Montgomery reduction (mont_mac2).  Block
// x = ciphertext + count * column block: the blocks of a batch that read the
// same plaintext tile run back to back and share it through L2.
template <int G, int V, int MINB>
__global__ void __launch_bounds__(256, MINB) k_pt_accum(const __grid_constant__ PtAccumDesc d) {
  const int r = blockIdx.y;
  const int c = blockIdx.x % d.count, xb = blockIdx.x / d.count;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t i = (static_cast<size_t>(xb) * blockDim.x + threadIdx.x) * V;
  if (i >= static_cast<size_t>(d.n)) return;
  const size_t idx = static_cast<size_t>(r) * d.n + i;
  const uint32_t qn = 0u - static_cast<uint32_t>(qi);
  uint32_t sb[G][V], sa[G][V];
#pragma unroll
  for (int o = 0; o < G; o++)
#pragma unroll
    for (int v = 0; v < V; v++) sb[o][v] = sa[o][v] = 0;
  // baby steps in pairs: two products per Montgomery reduction
  int t = 0;
  for (; t + 1 < d.ins; t += 2) {
    uint32_t xb0[V], xa0[V], xb1[V], xa1[V];
    ld_vec<V>(d.in_b[c][t] + idx, xb0);
    ld_vec<V>(d.in_a[c][t] + idx, xa0);
    ld_vec<V>(d.in_b[c][t + 1] + idx, xb1);
    ld_vec<V>(d.in_a[c][t + 1] + idx, xa1);
#pragma unroll
    for (int o = 0; o < G; o++) {
      if (o >= d.outs) continue;
      const uint32_t *p0 = d.pt[o][t], *p1 = d.pt[o][t + 1];
      if (p0 != nullptr && p1 != nullptr) {
        uint32_t m0[V], m1[V];
        ld_vec<V>(p0 + idx, m0);
        ld_vec<V>(p1 + idx, m1);
#pragma unroll
        for (int v = 0; v < V; v++) {
          sb[o][v] = add_mod(sb[o][v], mont_mac2(xb0[v], m0[v], xb1[v], m1[v], q, qn), q);
          sa[o][v] = add_mod(sa[o][v], mont_mac2(xa0[v], m0[v], xa1[v], m1[v], q, qn), q);
        }
      } else if (p0 != nullptr || p1 != nullptr) {
        const bool first = p0 != nullptr;
        uint32_t m[V];
        ld_vec<V>((first ? p0 : p1) + idx, m);
#pragma unroll
        for (int v = 0; v < V; v++) {
          sb[o][v] = add_mod(sb[o][v], mont_mul(first ? xb0[v] : xb1[v], m[v], q, qi), q);
          sa[o][v] = add_mod(sa[o][v], mont_mul(first ? xa0[v] : xa1[v], m[v], q, qi), q);
        }
      }
    }
  }
  if (t < d.ins) {
    uint32_t xb_[V], xa_[V];
    ld_vec<V>(d.in_b[c][t] + idx, xb_);
    ld_vec<V>(d.in_a[c][t] + idx, xa_);
#pragma unroll
    for (int o = 0; o < G; o++) {
      const uint32_t *p = d.pt[o][t];
      if (o < d.outs && p != nullptr) {
        uint32_t m[V];
        ld_vec<V>(p + idx, m);
#pragma unroll
        for (int v = 0; v < V; v++) {
          sb[o][v] = add_mod(sb[o][v], mont_mul(xb_[v], m[v], q, qi), q);
          sa[o][v] = add_mod(sa[o][v], mont_mul(xa_[v], m[v], q, qi), q);
        }
      }
    }
  }
#pragma unroll
  for (int o = 0; o < G; o++)
    if (o < d.outs) {
      st_vec<V>(d.out_b[c][o] + idx, sb[o]);
      st_vec<V>(d.out_a[c][o] + idx, sa[o]);
    }
}

// dst[p][r] = sum_t c[t][r] * src[t][p][r]  (Montgomery constants, canonical),
// 4 coefficients per thread in 16-byte vectors
__global__ void __launch_bounds__(256) k_const_accum(const __grid_constant__ ConstAccumDesc d) {
  const int r = blockIdx.y;
  const int part = blockIdx.z;
  const uint32_t q = d.q[r];
  const int32_t qi = d.qinv[r];
  const size_t n = static_cast<size_t>(d.n);
  const size_t i = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
  if (i >= n) return;
  uint32_t s[4] = {0, 0, 0, 0};
  for (int t = 0; t < d.terms; t++) {
    const uint32_t *src = d.src[t][part];
    if (!src) continue;
    uint32_t x[4];
    ld_vec<4>(src + static_cast<size_t>(d.src_row0[t] + r) * n + i, x);
    const uint32_t c = d.c[t][r];
#pragma unroll
    for (int l = 0; l < 4; l++) s[l] = add_mod(s[l], mont_mul(x[l], c, q, qi), q);
  }
  st_vec<4>(d.dst[part] + static_cast<size_t>(r) * n + i, s);
}

}  // namespace

void launch_modup_to_max(const ModUpToMaxDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.parts <= 0) return;
  k_modup_to_max<<<dim3(64, d.rows, d.parts), 256, 0, s>>>(d);
}

namespace {
// The faster of two launch variants of a shape: cached per (device, shape);
// the first launch of a shape outside a stream capture times both three
// times, interleaved, after a warm-up (every launch writes the same words);
// returns the variant the caller launches once more.
std::mutex g_pt_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_pt_cache;

template <class F>
int pick_variant(std::tuple<int, int, int, int> shape, F &&launch, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::tuple_cat(std::make_tuple(dev), shape);
  {
    std::lock_guard<std::mutex> lock(g_pt_mu);
    auto it = g_pt_cache.find(key);
    if (it != g_pt_cache.end()) return it->second;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return 0;
  constexpr int kReps = 3;
  cudaEvent_t ev[2 * kReps + 1] = {};
  for (auto &e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      for (auto &f : ev)
        if (f) cudaEventDestroy(f);
      return 0;
    }
  launch(0);
  launch(1);
  cudaEventRecord(ev[0], s);
  for (int r = 0; r < kReps; r++)
    for (int v = 0; v < 2; v++) {
      launch(v);
      cudaEventRecord(ev[2 * r + v + 1], s);
    }
  bool ok = cudaEventSynchronize(ev[2 * kReps]) == cudaSuccess;
  float best[2] = {1e30f, 1e30f};
  for (int r = 0; ok && r < kReps; r++)
    for (int v = 0; ok && v < 2; v++) {
      float t = 0.f;
      ok = cudaEventElapsedTime(&t, ev[2 * r + v], ev[2 * r + v + 1]) == cudaSuccess;
      best[v] = t < best[v] ? t : best[v];
    }
  for (auto &e : ev) cudaEventDestroy(e);
  const int pick = ok && best[1] < best[0] ? 1 : 0;
  if (ok) {
    std::lock_guard<std::mutex> lock(g_pt_mu);
    g_pt_cache[key] = pick;
  }
  return pick;
}
}  // namespace

void launch_pt_accum(const PtAccumDesc &d, cudaStream_t s, bool tune) {
  if (d.rows <= 0 || d.rows > 64 || d.outs <= 0 || d.outs > kMaxPtAccumOuts || d.ins <= 0 ||
      d.ins > kMaxPtAccumIn || d.count <= 0 || d.count > kMaxPtAccumCts)
    return;
  // vector width: every pointer 16-byte aligned and N a multiple of 4
  uintptr_t bits = static_cast<uintptr_t>(d.n) * 4;
  for (int c = 0; c < d.count; c++) {
    for (int t = 0; t < d.ins; t++)
      bits |= reinterpret_cast<uintptr_t>(d.in_b[c][t]) | reinterpret_cast<uintptr_t>(d.in_a[c][t]);
    for (int o = 0; o < d.outs; o++)
      bits |= reinterpret_cast<uintptr_t>(d.out_b[c][o]) | reinterpret_cast<uintptr_t>(d.out_a[c][o]);
  }
  for (int o = 0; o < d.outs; o++)
    for (int t = 0; t < d.ins; t++) bits |= reinterpret_cast<uintptr_t>(d.pt[o][t]);
  const bool vec = (bits & 15) == 0;
  auto grid = [&](int v) { return dim3(d.count * ((d.n / v + 255) / 256), d.rows); };
  if (!vec) {
    k_pt_accum<16, 1, 4><<<grid(1), 256, 0, s>>>(d);
  } else if (d.outs <= 4) {
    // 3 CTAs per SM (74 registers) or 4 (64, a few words spilled): timed
    // on the first launch of a shape when tuning
    auto launch = [&](int variant) {
      if (variant == 1)
        k_pt_accum<4, 4, 4><<<grid(4), 256, 0, s>>>(d);
      else
        k_pt_accum<4, 4, 3><<<grid(4), 256, 0, s>>>(d);
    };
    launch(tune ? pick_variant(std::make_tuple(d.count, d.rows, d.ins, d.outs), launch, s) : 0);
  } else if (d.outs <= 8) {
    k_pt_accum<8, 2, 4><<<grid(2), 256, 0, s>>>(d);
  } else {
    k_pt_accum<16, 1, 4><<<grid(1), 256, 0, s>>>(d);
  }
}

void launch_const_accum(const ConstAccumDesc &d, cudaStream_t s) {
  if (d.rows <= 0 || d.parts <= 0 || d.parts > kMaxConstAccumOuts || d.terms <= 0) return;
  k_const_accum<<<dim3((d.n / 4 + 255) / 256, d.rows, d.parts), 256, 0, s>>>(d);
}

}  // namespace chd
