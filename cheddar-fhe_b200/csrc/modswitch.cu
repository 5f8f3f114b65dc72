// Fused ModSwitch column kernel for N = 2^16.
//
// ModUp and ModDown (src/core/ModSwitch.cu:429-684 of the reference) are
//   INTT(sources) * (N q-hat_k)^-1 (centred)  ->  BConv  ->  NTT(targets).
// With the 128 x 512 limb layout used by ntt.cu, the INTT's last phase, the
// base conversion and the NTT's first phase all act on the same columns, so
// one CTA can take a 16-column tile through all three without touching HBM
// in between: the K centred sources of the tile stay in shared memory
// (K x 8 KB) and every target is converted, transformed and written once.
// The row phases before (INTT) and after (NTT, with the ModDown epilogue)
// stay in ntt.cu.
//
// Per tile and thread: 16 elements of one column.  The column transforms use
// the same stage schedule as ntt.cu (radix-16 on rows rg + 8k in registers,
// radix-8 on rows 8j + u after one shared-memory exchange).
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "arith.cuh"
#include "colpass.cuh"
#include "kernels.h"
#include "ntt_common.cuh"

namespace chd {
namespace {

// KMAX sources live in shared memory; with KR > 0 the sources KMAX ..
// KMAX + KR - 1 stay in registers (so that K = 13, 14 do not need
// the shared memory, and the lower occupancy, of the next larger KMAX).
template <int KMAX, int KR>
__global__ void __launch_bounds__(128, KMAX <= 8 ? 3 : 2) k_modswitch_cols(const __grid_constant__ MSColBatch b) {
  extern __shared__ uint32_t smem[];
  const MSColJob &jb = b.jobs[blockIdx.y];
  uint32_t *ex = smem;
  // centred sources, private to the thread that produced them:
  // xs4[(k * 4 + e / 4) * 128 + thread] holds elements 4(e/4) .. 4(e/4)+3
  int4 *xs4 = reinterpret_cast<int4 *>(smem + kExRows * kTC);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int cl = lane & 15, rg = 2 * w + (lane >> 4);
  const int col = blockIdx.x * kTC + cl;
  const int K = jb.K;
  const int Ks = K < KMAX ? K : KMAX;  // sources in shared memory
  int32_t xr[KR > 0 ? KR : 1][16];     // sources in registers

  // ---- phase A: INTT column stages, output constant, centring -> xs
  for (int k = 0; k < K; k++) {
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
    int32_t v[16];
#pragma unroll
    for (int e = 0; e < 16; e++) v[e] = centre(reduce2q(shoup_lazy(x[e], c0, c0s, q), q), q);
    if (k < KMAX) {
#pragma unroll
      for (int e4 = 0; e4 < 4; e4++)
        xs4[(k * 4 + e4) * 128 + t] = make_int4(v[4 * e4], v[4 * e4 + 1], v[4 * e4 + 2], v[4 * e4 + 3]);
    } else {
#pragma unroll
      for (int r = 0; r < KR; r++)
        if (k == KMAX + r)
#pragma unroll
          for (int e = 0; e < 16; e++) xr[r][e] = v[e];
    }
    __syncthreads();
  }
  // register sources of target row T: one more Montgomery chunk (at most 4 terms)
  auto reg_part = [&](const int32_t *T, uint32_t p, int32_t pinv, uint32_t (&v)[16]) {
    if (KR > 0 && K > KMAX) {
      int64_t a[16];
#pragma unroll
      for (int e = 0; e < 16; e++) a[e] = 0;
#pragma unroll
      for (int r = 0; r < KR; r++) {
        if (KMAX + r < K) {
          const int64_t tk = __ldg(T + KMAX + r);
#pragma unroll
          for (int e = 0; e < 16; e++) a[e] += static_cast<int64_t>(xr[r][e]) * tk;
        }
      }
#pragma unroll
      for (int e = 0; e < 16; e++) v[e] = add_mod(v[e], mont_reduce(a[e], p, pinv), p);
    }
  };

  // ---- phase B: exact BConv per target, then NTT column stages.  Targets
  // go in pairs: the two BConv accumulations share the source loads from
  // shared memory, and the two radix-16 column stages are independent
  // instruction streams (the kernel is latency-bound at 2-3 warps per
  // scheduler); the radix-8 stages then pass through the exchange buffer
  // one target after the other.
  auto bconv = [&](int m, uint32_t (&v)[16]) {
    const int g = jb.dst_gidx[m];
    const uint32_t p = __ldg(b.primes + g);
    const int32_t pinv = __ldg(b.qinvs + g);
    const int32_t *T = jb.table + m * K;
#pragma unroll
    for (int e = 0; e < 16; e++) v[e] = 0;
#pragma unroll
    for (int k0 = 0; k0 < KMAX; k0 += 4) {
      if (k0 < Ks) {
        int64_t a[16];
#pragma unroll
        for (int e = 0; e < 16; e++) a[e] = 0;
#pragma unroll
        for (int k = k0; k < k0 + 4; k++) {
          if (k < Ks) {
            const int64_t tk = __ldg(T + k);
#pragma unroll
            for (int e4 = 0; e4 < 4; e4++) {
              const int4 xv = xs4[(k * 4 + e4) * 128 + t];
              a[4 * e4] += static_cast<int64_t>(xv.x) * tk;
              a[4 * e4 + 1] += static_cast<int64_t>(xv.y) * tk;
              a[4 * e4 + 2] += static_cast<int64_t>(xv.z) * tk;
              a[4 * e4 + 3] += static_cast<int64_t>(xv.w) * tk;
            }
          }
        }
#pragma unroll
        for (int e = 0; e < 16; e++) v[e] = add_mod(v[e], mont_reduce(a[e], p, pinv), p);
      }
    }
    reg_part(T, p, pinv, v);
  };
  auto bconv2 = [&](int m0, int m1, uint32_t (&v0)[16], uint32_t (&v1)[16]) {
    const int g0 = jb.dst_gidx[m0], g1 = jb.dst_gidx[m1];
    const uint32_t p0 = __ldg(b.primes + g0), p1 = __ldg(b.primes + g1);
    const int32_t pi0 = __ldg(b.qinvs + g0), pi1 = __ldg(b.qinvs + g1);
    const int32_t *T0 = jb.table + m0 * K, *T1 = jb.table + m1 * K;
#pragma unroll
    for (int e = 0; e < 16; e++) v0[e] = v1[e] = 0;
#pragma unroll
    for (int k0 = 0; k0 < KMAX; k0 += 4) {
      if (k0 < Ks) {
        int64_t a0[16], a1[16];
#pragma unroll
        for (int e = 0; e < 16; e++) a0[e] = a1[e] = 0;
#pragma unroll
        for (int k = k0; k < k0 + 4; k++) {
          if (k < Ks) {
            const int64_t t0 = __ldg(T0 + k), t1 = __ldg(T1 + k);
#pragma unroll
            for (int e4 = 0; e4 < 4; e4++) {
              const int4 xv = xs4[(k * 4 + e4) * 128 + t];
              a0[4 * e4] += static_cast<int64_t>(xv.x) * t0;
              a1[4 * e4] += static_cast<int64_t>(xv.x) * t1;
              a0[4 * e4 + 1] += static_cast<int64_t>(xv.y) * t0;
              a1[4 * e4 + 1] += static_cast<int64_t>(xv.y) * t1;
              a0[4 * e4 + 2] += static_cast<int64_t>(xv.z) * t0;
              a1[4 * e4 + 2] += static_cast<int64_t>(xv.z) * t1;
              a0[4 * e4 + 3] += static_cast<int64_t>(xv.w) * t0;
              a1[4 * e4 + 3] += static_cast<int64_t>(xv.w) * t1;
            }
          }
        }
#pragma unroll
        for (int e = 0; e < 16; e++) {
          v0[e] = add_mod(v0[e], mont_reduce(a0[e], p0, pi0), p0);
          v1[e] = add_mod(v1[e], mont_reduce(a1[e], p1, pi1), p1);
        }
      }
    }
    reg_part(T0, p0, pi0, v0);
    reg_part(T1, p1, pi1, v1);
  };
  // radix-8 row groups of one target from the exchange buffer to HBM
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
  int m = 0;
  for (; m + 1 < jb.M; m += 2) {
    uint32_t v0[16], v1[16];
    bconv2(m, m + 1, v0, v1);
    {
      const uint32_t p0 = __ldg(b.primes + jb.dst_gidx[m]), p1 = __ldg(b.primes + jb.dst_gidx[m + 1]);
      const uint2 *tw0 = b.tw + (static_cast<size_t>(jb.dst_gidx[m]) << 16);
      const uint2 *tw1 = b.tw + (static_cast<size_t>(jb.dst_gidx[m + 1]) << 16);
      radix16_cols_fwd(v0, tw0, p0);  // stages m = 1, 2, 4, 8 on rows rg + 8e
      radix16_cols_fwd(v1, tw1, p1);
    }
    finish(m, v0);
    finish(m + 1, v1);
  }
  if (m < jb.M) {
    uint32_t v[16];
    bconv(m, v);
    const uint2 *tw = b.tw + (static_cast<size_t>(jb.dst_gidx[m]) << 16);
    radix16_cols_fwd(v, tw, __ldg(b.primes + jb.dst_gidx[m]));
    finish(m, v);
  }
}

}  // namespace

size_t modswitch_cols_smem(int kmax) { return (static_cast<size_t>(kExRows) * kTC + static_cast<size_t>(kmax) * 128 * kTC) * 4; }

namespace {

void launch_engine(const MSColBatch &b, int engine, int max_k, cudaStream_t s) {
  if ((engine == 3 || engine == 4) && modswitch_cols_tc8_supports(max_k)) {
    launch_modswitch_cols_tc8(b, max_k, engine == 4, s);
    return;
  }
  if (engine == 1 || engine == 3 || engine == 4) {
    launch_modswitch_cols_tc(b, max_k, s);
    return;
  }
  const dim3 grid(512 / kTC, b.count);
  auto go = [&](auto kern, int kmax) {
    const size_t sm = modswitch_cols_smem(kmax);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    kern<<<grid, 128, sm, s>>>(b);
  };
  // K = 9 stays with KMAX = 12: at 3 CTAs per SM (KMAX = 8 and one
  // register source) the 168-register cap and the second wave of a
  // 512-CTA grid cost more than the occupancy gains
  if (max_k <= 8)
    go(k_modswitch_cols<8, 0>, 8);
  else if (max_k <= 12)
    go(k_modswitch_cols<12, 0>, 12);
  else if (max_k <= 14)
    go(k_modswitch_cols<12, 2>, 12);
  else
    go(k_modswitch_cols<16, 0>, 16);
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Launches b with every job's targets spread over `groups` sub-jobs (each
// repeats its job's INTT column stages for its own subset of targets, at
// least 4 targets each): more, smaller CTAs for launches that would leave
// SMs idle.
void launch_split(const MSColBatch &b, int groups, int engine, int max_k, cudaStream_t s) {
  if (groups <= 1) {
    launch_engine(b, engine, max_k, s);
    return;
  }
  MSColBatch e = b;
  e.count = 0;
  for (int j = 0; j < b.count; j++) {
    const MSColJob &src = b.jobs[j];
    for (int g = 0; g < groups; g++) {
      const int m0 = src.M * g / groups, m1 = src.M * (g + 1) / groups;
      if (m1 <= m0) continue;
      MSColJob &d = e.jobs[e.count++];
      d = src;
      d.M = m1 - m0;
      d.table = src.table + static_cast<size_t>(m0) * src.K;
      for (int m = 0; m < d.M; m++) {
        d.dst_row[m] = src.dst_row[m0 + m];
        d.dst_gidx[m] = src.dst_gidx[m0 + m];
      }
      if (e.count == kMaxMSColJobs) {
        launch_engine(e, engine, max_k, s);
        e.count = 0;
      }
    }
  }
  if (e.count) launch_engine(e, engine, max_k, s);
}

// the split of the fixed engines: about two CTAs per SM, at least 4 targets
// per sub-job
int heuristic_groups(const MSColBatch &b, int max_m) {
  const int tiles = 512 / kTC;
  const int want = 2 * sm_count();
  int groups = (want + tiles * b.count - 1) / (tiles * b.count);
  groups = groups < 1 ? 1 : groups;
  const int by_m = max_m / 4 > 1 ? max_m / 4 : 1;
  return groups > by_m ? by_m : groups;
}

// Autotuning (engine 2, CHD_BCONV_AUTO): which engine and tile and which
// target split are fastest depends on the launch (the CUDA-core pass wins
// when a launch holds one ciphertext's few jobs, the tensor-core passes on
// batches; small launches gain from the split).  The first launch of a shape
// (device, largest K, jobs, largest M) outside a stream capture times every
// candidate (engine and tile in {CUDA cores, tensor cores with 128-thread
// tiles, tensor cores with 256-thread tiles for K <= 12 at 80 or, for
// K <= 8, 128 registers per thread} x split in
// {1, 2, 4, heuristic}) three times after a
// warm-up, interleaved, with CUDA events (a host synchronisation, once per
// shape), keeps the fastest launch and caches the choice for the process.
// Every candidate writes identical residues, so the tuning launches leave
// the right outputs.  During a capture an untuned shape uses the tensor
// cores with the heuristic split.  Returns true when the tuning launches
// have done the work; *engine and *groups receive the choice otherwise.
struct Choice {
  int engine, groups;
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, Choice> g_tune_cache;

bool tune_and_launch(const MSColBatch &b, int max_k, int max_m, cudaStream_t s, Choice *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, max_k, b.count, max_m);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      *out = it->second;
      return false;
    }
  }
  const int hg = heuristic_groups(b, max_m);
  *out = Choice{1, hg};
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
  std::vector<Choice> cand;
  const int by_m = max_m / 4 > 1 ? max_m / 4 : 1;
  for (int e : {0, 1, 3, 4})
    for (int g : {1, 2, 4, hg})
      if (g <= by_m) {
        bool seen = false;
        for (const Choice &c : cand) seen |= c.engine == e && c.groups == g;
        // engine 4 differs from 3 only for K <= 8
        const bool valid = e < 3 || (modswitch_cols_tc8_supports(max_k) && (e == 3 || max_k <= 8));
        if (!seen && valid) cand.push_back(Choice{e, g});
      }
  constexpr int kRounds = 3;
  const int nc = static_cast<int>(cand.size());
  std::vector<cudaEvent_t> ev(nc * kRounds + 1, nullptr);
  for (auto &x : ev)
    if (cudaEventCreate(&x) != cudaSuccess) {
      for (auto &f : ev)
        if (f) cudaEventDestroy(f);
      return false;
    }
  for (const Choice &c : cand) launch_split(b, c.groups, c.engine, max_k, s);  // warm-up
  cudaEventRecord(ev[0], s);
  for (int r = 0; r < kRounds; r++)
    for (int i = 0; i < nc; i++) {
      launch_split(b, cand[i].groups, cand[i].engine, max_k, s);
      cudaEventRecord(ev[r * nc + i + 1], s);
    }
  bool ok = cudaEventSynchronize(ev.back()) == cudaSuccess;
  std::vector<float> best(nc, 1e30f);
  for (int r = 0; ok && r < kRounds; r++)
    for (int i = 0; ok && i < nc; i++) {
      float t = 0.f;
      ok = cudaEventElapsedTime(&t, ev[r * nc + i], ev[r * nc + i + 1]) == cudaSuccess;
      best[i] = t < best[i] ? t : best[i];
    }
  for (auto &x : ev) cudaEventDestroy(x);
  if (ok) {
    int bi = 0;
    for (int i = 1; i < nc; i++)
      if (best[i] < best[bi]) bi = i;
    // timed alone, a CUDA-core candidate can edge out a tensor-core one by
    // noise; but the CUDA-core pass (168-254 registers per thread) shares an
    // SM poorly with the kernels of a key switch's other half on the second
    // stream, so within 3 % of the fastest the fastest tensor-core candidate
    // is kept
    if (cand[bi].engine == 0) {
      int ti = -1;
      for (int i = 0; i < nc; i++)
        if (cand[i].engine != 0 && best[i] <= best[bi] * 1.03f && (ti < 0 || best[i] < best[ti])) ti = i;
      if (ti >= 0) bi = ti;
    }
    *out = cand[bi];
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = cand[bi];
  }
  return true;
}

}  // namespace

void launch_modswitch_cols(const MSColBatch &b, int log_n, cudaStream_t s) {
  if (b.count <= 0 || log_n != 16) return;
  int max_k = 0, max_m = 0;
  for (int j = 0; j < b.count; j++) {
    max_k = b.jobs[j].K > max_k ? b.jobs[j].K : max_k;
    max_m = b.jobs[j].M > max_m ? b.jobs[j].M : max_m;
  }
  if (b.engine == 2) {
    Choice c{1, 1};
    if (tune_and_launch(b, max_k, max_m, s, &c)) return;
    launch_split(b, c.groups, c.engine, max_k, s);
    return;
  }
  launch_split(b, heuristic_groups(b, max_m), b.engine, max_k, s);
}

int modswitch_tuned_shapes(int *out, int cap) {
  // (device, max_k, jobs, max_m, engine, groups) per cached shape
  std::lock_guard<std::mutex> lock(g_tune_mu);
  int k = 0;
  for (const auto &kv : g_tune_cache) {
    if (out && k < cap) {
      int *o = out + 6 * k;
      o[0] = std::get<0>(kv.first);
      o[1] = std::get<1>(kv.first);
      o[2] = std::get<2>(kv.first);
      o[3] = std::get<3>(kv.first);
      o[4] = kv.second.engine;
      o[5] = kv.second.groups;
    }
    k++;
  }
  return k;
}

}  // namespace chd
