// Linear transforms with double hoisting (baby-step / giant-step), the
// evaluation engine of CoeffToSlot and SlotToCoeff.
//
// Planning (host, FP64) follows the reference step by step:
//   StripedMatrix::Mult (src/extension/StripedMatrix.cpp:16-48),
//   LinearTransform::DetermineStride / ConstructPlainHoistMap
//   (src/extension/LinearTransform.cpp:8-75), the baby/giant swap of the
//   HoistHandler constructor and CompilePlaintexts (src/extension/Hoist.cu:
//   120-167: every diagonal encoded at pt_level with the alpha auxiliary
//   primes).
// Evaluation (device) computes the same formula as HoistHandler::Evaluate
// (Hoist.cu:554-975):
//   baby steps   bs_r = Permute_r(ModUp(a) (.) key_r + P b)     (Q u P, one launch)
//                bs_0 = P (b, a)                               (Q u P, aux rows 0)
//   giant steps  acc_g = sum_r pt_(g,r) (.) bs_r
//                out   = acc_0 + sum_g Permute_g(KeyMult_g(ModUp(ModDown(acc_g.a))))
//                        + sum_g Permute_g((acc_g.b, 0))
//                res   = ModDownAndRescale(out)
// and, when the map has the single giant step 0 (swapped to baby steps
// only),
//                out   = P (b, a) (.) pt_0 + sum_r Permute_r((KeyMult_r(ModUp(a)) + (P b, 0)) (.) pt_r).
// Every step is exact modular arithmetic, so any evaluation order gives
// the reference's residues.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>

#include "host.h"
#include "kernels.h"

namespace chd {

using cd = std::complex<double>;

SMat smat_mult(const SMat &a, const SMat &b) {
  // StripedMatrix::Mult(a, b), StripedMatrix.cpp:16-38
  const int w = a.w;
  SMat c;
  c.h = c.w = w;
  for (const auto &da : a.d)
    for (const auto &db : b.d) {
      const int i = da.first, dest = (da.first + db.first) % w;
      auto it = c.d.find(dest);
      if (it == c.d.end()) it = c.d.emplace(dest, std::vector<cd>(w)).first;
      std::vector<cd> &dc = it->second;
      const std::vector<cd> &x = da.second, &y = db.second;
      for (int k = 0; k < w; k++) dc[k] += x[k] * y[(k + i) % w];
    }
  return c;
}

SMat smat_scale(const SMat &a, cd b) {
  // StripedMatrix::Mult(a, Complex), StripedMatrix.cpp:40-48
  SMat c;
  c.h = a.h;
  c.w = a.w;
  for (const auto &da : a.d) {
    std::vector<cd> v(da.second.size());
    for (size_t j = 0; j < v.size(); j++) v[j] = da.second[j] * b;
    c.d.emplace(da.first, std::move(v));
  }
  return c;
}

namespace {

int gcd_int(int a, int b) {
  while (b) {
    const int t = a % b;
    a = b;
    b = t;
  }
  return a;
}

}  // namespace

Status Context::lt_build(const SMat &m, int pt_level, double pt_scale, int bs, int gs, int pre_rotation,
                         int additional_pt_rot, bool suppress_swap, LTPlan *out) {
  CHD_CHECK(m.h == m.w && m.w > 0 && (m.w & (m.w - 1)) == 0, kErrInvalidArg,
            "LinearTransform requires a square power-of-two matrix");
  CHD_CHECK(m.w <= P->n / 2, kErrInvalidArg, "LinearTransform: matrix wider than N/2 slots");
  CHD_CHECK(pt_level >= 1 && pt_level <= P->max_level, kErrInvalidLevel, "LinearTransform: invalid level");
  for (auto &p : out->pts) cudaFree(p.dev);
  *out = LTPlan{};
  LTPlan &pl = *out;
  pl.pt_level = pt_level;
  pl.pt_scale = pt_scale;
  pl.width = m.w;
  const int w = m.w;
  // DetermineStride, LinearTransform.cpp:8-36
  int g = 0, max_rot = 0, num_pt = 0;
  for (const auto &d : m.d) {
    num_pt++;
    int rot = (d.first - pre_rotation) % w;
    if (rot < 0) rot += w;
    g = (g == 0 && rot == 0) ? rot : gcd_int(g, rot);
    max_rot = std::max(max_rot, rot);
  }
  CHD_CHECK(num_pt > 1, kErrInvalidArg, "LinearTransform requires at least 2 plaintexts");
  CHD_CHECK(g > 0, kErrInvalidArg, "LinearTransform: no non-zero rotation");
  CHD_CHECK(max_rot <= (bs * gs - 1) * g, kErrInvalidArg, "LinearTransform: matrix does not fit bs x gs");
  const int stride = g;
  // ConstructPlainHoistMap, LinearTransform.cpp:38-75
  std::map<int, std::map<int, std::vector<cd>>> hm;
  const int gs_stride = stride * bs;
  for (const auto &d : m.d) {
    int rot = (d.first - pre_rotation) % w;
    if (rot < 0) rot += w;
    const int bs_rot = rot % gs_stride, gs_rot = rot - bs_rot;
    std::vector<cd> &v = hm[gs_rot].emplace(bs_rot, std::vector<cd>(w, cd(0, 0))).first->second;
    int off = (gs_rot - additional_pt_rot) % w;
    if (off < 0) off += w;
    for (int j = 0; j < w; j++) v[(j + off) % w] = d.second[j];
  }
  // HoistHandler constructor, Hoist.cu:146-166: one giant step 0 -> baby steps
  // become giant steps (pre-shifted messages)
  if (hm.size() == 1 && hm.begin()->first == 0 && !suppress_swap) {
    std::map<int, std::map<int, std::vector<cd>>> sw;
    for (const auto &e : hm.begin()->second) {
      const int sz = static_cast<int>(e.second.size());
      std::vector<cd> v(sz);
      for (int i = 0; i < sz; i++) v[(i + e.first) % sz] = e.second[i];
      sw[e.first].emplace(0, std::move(v));
    }
    hm.swap(sw);
  }
  for (const auto &gsm : hm)
    for (const auto &b : gsm.second) pl.bs_idx.push_back(b.first);
  std::sort(pl.bs_idx.begin(), pl.bs_idx.end());
  pl.bs_idx.erase(std::unique(pl.bs_idx.begin(), pl.bs_idx.end()), pl.bs_idx.end());
  // CompilePlaintexts, Hoist.cu:130-145
  const NP np = P->level_np(pt_level, P->alpha);
  const size_t words = static_cast<size_t>(np.total()) * P->n;
  for (const auto &gsm : hm) {
    pl.gs_idx.push_back(gsm.first);
    for (const auto &b : gsm.second) {
      LTPlan::Pt pt;
      pt.gs = gsm.first;
      pt.bs = b.first;
      pt.msg = b.second;
      if (cudaMalloc(&pt.dev, words * 4) != cudaSuccess) {
        set_error("LinearTransform: plaintext allocation failed");
        return kErrAlloc;
      }
      pl.pts.push_back(std::move(pt));
      LTPlan::Pt &p = pl.pts.back();
      int ns = 0;
      CHD_TRY(encode(pt_level, pt_scale, p.msg.data(), static_cast<int>(p.msg.size()), P->alpha, p.dev, &ns));
      pl.pt_slots = std::max(pl.pt_slots, ns);
    }
  }
  return kOk;
}

LTPlan::~LTPlan() {
  for (auto &p : pts) cudaFree(p.dev);
}

Status lt_min_ks_strides(const LTPlan &pl, int *bs_stride, int *gs_stride) {
  // HoistHandler::CheckStrideMinKS, Hoist.cu:169-205: non-zero baby (giant)
  // steps must be 1..k times their gcd
  auto stride = [](const std::vector<int> &idx, int *out) -> bool {
    int g = 0, cnt = 0, mx = 0;
    for (int x : idx) {
      if (x == 0) continue;
      int a = g, b = x;
      while (b) {
        const int t = a % b;
        a = b;
        b = t;
      }
      g = a;
      cnt++;
      mx = std::max(mx, x);
    }
    *out = g;
    return cnt * g == mx;
  };
  CHD_CHECK(stride(pl.bs_idx, bs_stride), kErrInvalidArg, "MinKS does not apply to the given hoist map baby-step sequence");
  CHD_CHECK(stride(pl.gs_idx, gs_stride), kErrInvalidArg, "MinKS does not apply to the given hoist map giant-step sequence");
  return kOk;
}

Status Context::lt_evaluate_min_ks(DeviceCt &res, const DeviceCt &in, const LTPlan &pl, const RotKeys &keys) {
  DeviceCt *r = &res;
  const DeviceCt *i = &in;
  return lt_evaluate_min_ks_batch(1, &r, &i, pl, keys);
}

Status Context::lt_evaluate_min_ks_batch(int count, DeviceCt *const *res, const DeviceCt *const *in,
                                         const LTPlan &pl, const RotKeys &keys) {
  // HoistHandler::EvaluateMinKSBabyStep / EvaluateMinKSGiantStep
  // (Hoist.cu:490-552): baby steps by repeated HRot with the baby stride,
  // giant steps in reverse order, accumulate, HRot by the giant stride,
  // then Rescale.  Works in the Q basis of pt_level.  Every rotation and the
  // final rescale run once over the `count` ciphertexts.
  const int level = pl.pt_level;
  const int n = P->n;
  for (int c = 0; c < count; c++) {
    CHD_CHECK(!in[c]->has_rx && in[c]->np.aux == 0, kErrShape, "Hoist: input should be relinearized and mod-down");
    CHD_CHECK(in[c]->np == P->level_np(level), kErrShape, "Hoist: input level mismatch");
  }
  CHD_CHECK(!(pl.bs_idx.size() == 1 && pl.bs_idx[0] == 0), kErrInvalidArg,
            "Hoist: min_ks should be false for bs == 1 case");
  int bs_stride = 0, gs_stride = 0;
  CHD_TRY(lt_min_ks_strides(pl, &bs_stride, &gs_stride));
  auto key_of = [&](int r) -> const DeviceEvk * {
    auto it = keys.find(r);
    return it == keys.end() ? nullptr : it->second;
  };
  const NP np = P->level_np(level);
  const int nq = np.q();
  const size_t bytes = static_cast<size_t>(nq) * n * 4;
  std::vector<int> g(nq);
  P->gidx(np, g.data());
  ArenaScope scope(arena);
  // baby steps in the Q basis
  std::vector<std::vector<DeviceCt>> bs(count);
  std::map<int, int> slot_of;
  for (size_t i = 0; i < pl.bs_idx.size(); i++) slot_of[pl.bs_idx[i]] = static_cast<int>(i);
  for (int c = 0; c < count; c++) {
    bs[c].resize(pl.bs_idx.size());
    for (size_t i = 0; i < pl.bs_idx.size(); i++) CHD_TRY(scratch_ct(arena, bs[c][i], np, false, n));
  }
  const DeviceEvk *kb = key_of(bs_stride);
  std::vector<DeviceCt *> dst(count);
  std::vector<const DeviceCt *> src(count);
  for (size_t i = 0; i < pl.bs_idx.size(); i++) {
    const int r = pl.bs_idx[i];
    if (r == 0) {
      for (int c = 0; c < count; c++) {
        cudaMemcpyAsync(bs[c][i].bx, in[c]->bx, bytes, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(bs[c][i].ax, in[c]->ax, bytes, cudaMemcpyDeviceToDevice, stream);
        bs[c][i].scale = in[c]->scale;
        bs[c][i].num_slots = in[c]->num_slots;
      }
    } else {
      CHD_CHECK(kb, kErrKey, "Hoist: missing rotation key " + std::to_string(bs_stride));
      auto it = slot_of.find(r - bs_stride);
      CHD_CHECK(it != slot_of.end(), kErrInvalidArg, "Hoist: MinKS baby-step sequence is not complete");
      for (int c = 0; c < count; c++) {
        dst[c] = &bs[c][i];
        src[c] = &bs[c][it->second];
      }
      CHD_TRY(hrot_batch(count, dst.data(), src.data(), *kb, bs_stride));
    }
  }
  // giant steps, reversed
  std::vector<DeviceCt> acc(count), tmp(count);
  for (int c = 0; c < count; c++) {
    CHD_TRY(scratch_ct(arena, acc[c], np, false, n));
    CHD_TRY(scratch_ct(arena, tmp[c], np, false, n));
  }
  const DeviceEvk *kg = key_of(gs_stride);
  bool first = true;
  int prev = 0;
  for (auto git = pl.gs_idx.rbegin(); git != pl.gs_idx.rend(); ++git) {
    const int gsi = *git;
    CHD_CHECK(first || prev == gsi + gs_stride, kErrInvalidArg, "Hoist: MinKS giant-step sequence is not complete");
    // this giant step's terms (shared) and each ciphertext's baby steps
    std::vector<int> in_slot;
    std::map<int, int> in_of;
    std::vector<const uint32_t *> pts;
    for (const auto &pt : pl.pts) {
      if (pt.gs != gsi) continue;
      CHD_CHECK(!in_of.count(pt.bs), kErrInvalidArg, "Hoist: a giant step names one baby step twice");
      CHD_CHECK(static_cast<int>(in_slot.size()) < kMaxPtAccumIn, kErrUnsupported, "Hoist: too many baby steps");
      in_of.emplace(pt.bs, static_cast<int>(in_slot.size()));
      in_slot.push_back(slot_of.at(pt.bs));
      pts.push_back(pt.dev);  // the first nq rows are the q primes
    }
    for (int c = 0; c < count && in_slot.empty(); c++) {  // no plaintexts: a zero sum
      DeviceCt &o = first ? acc[c] : tmp[c];
      cudaMemsetAsync(o.bx, 0, static_cast<size_t>(nq) * n * 4, stream);
      cudaMemsetAsync(o.ax, 0, static_cast<size_t>(nq) * n * 4, stream);
    }
    for (int c0 = 0; c0 < count && !in_slot.empty(); c0 += kMaxPtAccumCts) {
      PtAccumDesc d{};
      d.count = std::min(kMaxPtAccumCts, count - c0);
      d.ins = static_cast<int>(in_slot.size());
      for (int k = 0; k < d.ins; k++) d.pt[0][k] = pts[k];
      for (int c = 0; c < d.count; c++) {
        for (int k = 0; k < d.ins; k++) {
          d.in_b[c][k] = bs[c0 + c][in_slot[k]].bx;
          d.in_a[c][k] = bs[c0 + c][in_slot[k]].ax;
        }
        DeviceCt &o = first ? acc[c0 + c] : tmp[c0 + c];
        d.out_b[c][0] = o.bx;
        d.out_a[c][0] = o.ax;
      }
      for (int r = 0; r < nq; r++) {
        d.q[r] = P->primes[g[r]];
        d.qinv[r] = P->qinv[g[r]];
      }
      d.rows = nq;
      d.n = n;
      d.outs = 1;
      launch_pt_accum(d, stream, ks_engine == 2);
    }
    for (int c = 0; c < count; c++) {
      if (!first) CHD_TRY(add(acc[c], acc[c], tmp[c]));
      acc[c].scale = in[c]->scale * pl.pt_scale;
      acc[c].num_slots = std::max(in[c]->num_slots, pl.pt_slots);
    }
    if (gsi != 0) {
      CHD_CHECK(kg, kErrKey, "Hoist: missing rotation key " + std::to_string(gs_stride));
      for (int c = 0; c < count; c++) {
        dst[c] = &tmp[c];
        src[c] = &acc[c];
      }
      CHD_TRY(hrot_batch(count, dst.data(), src.data(), *kg, gs_stride));
      for (int c = 0; c < count; c++) {
        cudaMemcpyAsync(acc[c].bx, tmp[c].bx, bytes, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(acc[c].ax, tmp[c].ax, bytes, cudaMemcpyDeviceToDevice, stream);
      }
    } else {
      CHD_CHECK(first || prev == gs_stride, kErrInvalidArg, "Hoist: MinKS giant-step sequence is not complete");
    }
    first = false;
    prev = gsi;
  }
  // final Rescale of every accumulator in one ModDown launch sequence
  std::vector<const uint32_t *> rsrc(2 * count);
  std::vector<uint32_t *> rdst(2 * count);
  for (int c = 0; c < count; c++) {
    CHD_TRY(res[c]->reserve(P->level_np(level - 1, 0), false, n));
    rsrc[2 * c] = acc[c].bx;
    rsrc[2 * c + 1] = acc[c].ax;
    rdst[2 * c] = res[c]->bx;
    rdst[2 * c + 1] = res[c]->ax;
  }
  CHD_TRY(moddown(level, MDType::kRescale, rsrc.data(), rdst.data(), 2 * count));
  for (int c = 0; c < count; c++) {
    res[c]->scale = acc[c].scale / P->rescale_prod[level];
    res[c]->num_slots = acc[c].num_slots;
  }
  return check_cuda("linear transform (min-KS)");
}

namespace {

// Row-level building blocks of the hoisted evaluation at one level (Q u P
// basis of that level), shared by the single and the batched paths.
struct HoistOps {
  Context &C;
  const int level, n;
  const NP qp;
  const int nq, tot, prime_offset;
  const LevelMS &m;
  std::vector<int> g;
  const size_t tw;  // words of one Q u P polynomial

  HoistOps(Context &c, int lvl)
      : C(c),
        level(lvl),
        n(c.P->n),
        qp(c.P->level_np(lvl, c.P->alpha)),
        nq(qp.q()),
        tot(qp.total()),
        prime_offset(c.P->max_ter - qp.ter),
        m(c.lms(lvl)),
        g(tot),
        tw(static_cast<size_t>(tot) * c.P->n) {
    c.P->gidx(qp, g.data());
  }
  // P * x on q rows, zero on aux rows (PseudoModUp + ZeroExtend)
  void pseudo_modup(const uint32_t *src, uint32_t *dst) const {
    ConstAccumDesc d{};
    d.terms = 1;
    d.src[0][0] = src;
    d.src_row0[0] = 0;
    d.dst[0] = dst;
    for (int r = 0; r < nq; r++) {
      d.q[r] = C.P->primes[g[r]];
      d.qinv[r] = C.P->qinv[g[r]];
      d.c[0][r] = C.p_prod[prime_offset + r];
    }
    d.rows = nq;
    d.parts = 1;
    d.n = n;
    launch_const_accum(d, C.stream);
    cudaMemsetAsync(dst + static_cast<size_t>(nq) * n, 0, static_cast<size_t>(tot - nq) * n * 4, C.stream);
  }
  // sum_i ModUp(x)_i (.) key_i over Q u P (MultKeyNoModDown, Context.cpp:610-648)
  // for `count` ciphertexts sharing the key: mu[c][digit]
  Status key_mult(int count, uint32_t *const *const *mu, const DeviceEvk &k, uint32_t *const *ob,
                  uint32_t *const *oa) const {
    if (!(k.np.aux == C.P->alpha && k.np.q() == C.P->L)) {
      set_error("Hoist: key basis mismatch");
      return kErrKey;
    }
    const size_t kstride = static_cast<size_t>(C.P->L + C.P->alpha) * n;
    for (int c0 = 0; c0 < count; c0 += kMaxKeyMacCts) {
      KeyMacDesc d{};
      int nb = 0;
      for (int i = 0; i < m.beta; i++) {
        if (m.dig_e[i] <= 0) continue;
        if (i >= k.beta) {
          set_error("Hoist: key has too few digits");
          return kErrKey;
        }
        d.kb[nb] = k.bx + i * kstride;
        d.ka[nb] = k.ax + i * kstride;
        nb++;
      }
      d.beta = nb;
      d.rows = tot;
      d.nq = nq;
      d.count = std::min(kMaxKeyMacCts, count - c0);
      for (int r = 0; r < tot; r++) {
        d.q[r] = C.P->primes[g[r]];
        d.qinv[r] = C.P->qinv[g[r]];
        d.p_prod[r] = 0;
        d.key_row[r] = static_cast<int16_t>(r < nq ? prime_offset + r : C.P->L + (r - nq));
      }
      for (int c = 0; c < d.count; c++) {
        int b = 0;
        for (int i = 0; i < m.beta; i++)
          if (m.dig_e[i] > 0) d.ct[c].mu[b++] = mu[c0 + c][i];
        d.ct[c].d0 = d.ct[c].d1 = nullptr;
        d.ct[c].acc_b = ob[c0 + c];
        d.ct[c].acc_a = oa[c0 + c];
      }
      launch_key_mac(d, C.P->log_n, C.stream);
    }
    return kOk;
  }
  // dst (+)= Permute_g(src) over the Q u P rows of one part
  void permute_rows(const uint32_t *src, uint32_t *dst, const uint32_t *add, int amount) const {
    PermuteBatch pb{};
    pb.galois = C.P->galois_of(amount);
    for (int r = 0; r < tot; r++) {
      if (pb.count == kMaxPermuteRows) {
        launch_permute(pb, C.P->log_n, C.stream);
        pb.count = 0;
      }
      PermuteRow &pr = pb.rows[pb.count++];
      pr.src = src + static_cast<size_t>(r) * n;
      pr.dst = dst + static_cast<size_t>(r) * n;
      pr.add = add ? add + static_cast<size_t>(r) * n : nullptr;
      pr.src2 = nullptr;
      pr.q = C.P->primes[g[r]];
    }
    launch_permute(pb, C.P->log_n, C.stream);
  }
  // dst_j += Permute_g(src_j + src2_j) over the Q u P rows of nparts parts
  // (src2_j may be null), the rows of all parts filling each launch
  void permute_add_many(int nparts, const uint32_t *const *src, const uint32_t *const *src2, uint32_t *const *dst,
                        int amount) const {
    PermuteBatch pb{};
    pb.galois = C.P->galois_of(amount);
    for (int j = 0; j < nparts; j++)
      for (int r = 0; r < tot; r++) {
        if (pb.count == kMaxPermuteRows) {
          launch_permute(pb, C.P->log_n, C.stream);
          pb.count = 0;
        }
        const size_t o = static_cast<size_t>(r) * n;
        PermuteRow &pr = pb.rows[pb.count++];
        pr.src = src[j] + o;
        pr.src2 = src2[j] ? src2[j] + o : nullptr;
        pr.dst = dst[j] + o;
        pr.add = dst[j] + o;
        pr.q = C.P->primes[g[r]];
      }
    launch_permute(pb, C.P->log_n, C.stream);
  }
  void add_rows(const uint32_t *a, const uint32_t *b, uint32_t *dst, int rows) const {
    ElemBatch eb{};
    for (int r = 0; r < rows; r++) {
      if (eb.count == kMaxElemRows) {
        launch_elementwise(ElemOp::kAdd, eb, C.P->log_n, C.stream);
        eb.count = 0;
      }
      ElemRow &e = eb.rows[eb.count++];
      e.a = a + static_cast<size_t>(r) * n;
      e.b = b + static_cast<size_t>(r) * n;
      e.dst = dst + static_cast<size_t>(r) * n;
      e.q = C.P->primes[g[r]];
      e.qinv = C.P->qinv[g[r]];
    }
    launch_elementwise(ElemOp::kAdd, eb, C.P->log_n, C.stream);
  }
  using Pairs = std::vector<std::pair<const uint32_t *, const uint32_t *>>;
  using OutPairs = std::vector<std::pair<uint32_t *, uint32_t *>>;
  // giant-step plaintext accumulation of `count` ciphertexts sharing the
  // plaintexts: outs[c][o] = sum over terms[o] of pt (.) ins[c][term]
  Status pt_accum(int count, const std::vector<Pairs> &ins,
                  const std::vector<std::vector<std::pair<int, const uint32_t *>>> &terms,
                  const std::vector<OutPairs> &outs) const {
    const int nin = static_cast<int>(ins[0].size());
    if (nin > kMaxPtAccumIn) {
      set_error("Hoist: too many baby steps");
      return kErrUnsupported;
    }
    const size_t nout = outs[0].size();
    for (int c0 = 0; c0 < count; c0 += kMaxPtAccumCts) {
      const int cn = std::min(kMaxPtAccumCts, count - c0);
      for (size_t o0 = 0; o0 < nout; o0 += kMaxPtAccumOuts) {
        PtAccumDesc d{};
        d.count = cn;
        d.ins = nin;
        for (int c = 0; c < cn; c++)
          for (int i = 0; i < nin; i++) {
            d.in_b[c][i] = ins[c0 + c][i].first;
            d.in_a[c][i] = ins[c0 + c][i].second;
          }
        for (int r = 0; r < tot; r++) {
          d.q[r] = C.P->primes[g[r]];
          d.qinv[r] = C.P->qinv[g[r]];
        }
        d.rows = tot;
        d.n = n;
        d.outs = static_cast<int>(std::min<size_t>(kMaxPtAccumOuts, nout - o0));
        for (int o = 0; o < d.outs; o++) {
          for (const auto &t : terms[o0 + o]) {
            if (t.first < 0 || t.first >= nin || d.pt[o][t.first]) {
              set_error("Hoist: a giant step names one baby step twice or one that does not exist");
              return kErrInvalidArg;
            }
            d.pt[o][t.first] = t.second;
          }
          for (int c = 0; c < cn; c++) {
            d.out_b[c][o] = outs[c0 + c][o0 + o].first;
            d.out_a[c][o] = outs[c0 + c][o0 + o].second;
          }
        }
        launch_pt_accum(d, C.stream, C.ks_engine == 2);
      }
    }
    return kOk;
  }
};

}  // namespace

Status Context::lt_evaluate(DeviceCt &res, const DeviceCt &in, const LTPlan &pl, const RotKeys &keys) {
  // HoistHandler::Evaluate, Hoist.cu:554-975 (non-min-KS, fused kernels)
  const bool only_gs = pl.bs_idx.size() == 1 && pl.bs_idx[0] == 0;
  if (!only_gs) {
    DeviceCt *r = &res;
    const DeviceCt *i = &in;
    return lt_evaluate_batch(1, &r, &i, pl, keys);
  }
  const int level = pl.pt_level;
  const int n = P->n;
  CHD_CHECK(!in.has_rx && in.np.aux == 0, kErrShape, "Hoist: input should be relinearized and mod-down");
  CHD_CHECK(in.np == P->level_np(level), kErrShape, "Hoist: input level mismatch");
  const HoistOps H(*this, level);
  const size_t tw_ = H.tw;
  auto key_of = [&](int r) -> const DeviceEvk * {
    auto it = keys.find(r);
    return it == keys.end() ? nullptr : it->second;
  };
  ArenaScope scope(arena);
  auto alloc = [&](size_t words) { return static_cast<uint32_t *>(arena.alloc(words * 4)); };
  std::vector<uint32_t *> mu(H.m.beta);
  for (int i = 0; i < H.m.beta; i++) {
    mu[i] = alloc(tw_);
    CHD_CHECK(mu[i], kErrAlloc, "Hoist: scratch allocation failed");
  }
  uint32_t *fb = alloc(tw_), *fa = alloc(tw_);  // final accumulator (Q u P)
  CHD_CHECK(fb && fa, kErrAlloc, "Hoist: scratch allocation failed");
  // Hoist.cu:706-808: ModUp(a) once, per giant step key mult + P b, times pt,
  // then PermuteAccum
  CHD_TRY(modup(level, in.ax, mu.data()));
  uint32_t *bxp = alloc(tw_), *tb = alloc(tw_), *ta = alloc(tw_);
  uint32_t *p0b = alloc(tw_), *p0a = alloc(tw_);
  CHD_CHECK(bxp && tb && ta && p0b && p0a, kErrAlloc, "Hoist: scratch allocation failed");
  H.pseudo_modup(in.bx, bxp);
  bool have0 = false;
  bool first_sum = true;
  for (const auto &pt : pl.pts) {
    if (pt.gs == 0) {
      H.pseudo_modup(in.ax, p0a);
      CHD_TRY(H.pt_accum(1, {{{bxp, p0a}}}, {{{0, pt.dev}}}, {{{fb, fa}}}));
      have0 = true;
    }
  }
  uint32_t *const *mu1[1] = {mu.data()};
  for (const auto &pt : pl.pts) {
    if (pt.gs == 0) continue;
    const DeviceEvk *k = key_of(pt.gs);
    CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(pt.gs));
    CHD_TRY(H.key_mult(1, mu1, *k, &tb, &ta));
    H.add_rows(tb, bxp, tb, H.nq);
    CHD_TRY(H.pt_accum(1, {{{tb, ta}}}, {{{0, pt.dev}}}, {{{p0b, p0a}}}));
    if (!have0 && first_sum) {
      H.permute_rows(p0b, fb, nullptr, pt.gs);
      H.permute_rows(p0a, fa, nullptr, pt.gs);
    } else {
      H.permute_rows(p0b, fb, fb, pt.gs);
      H.permute_rows(p0a, fa, fa, pt.gs);
    }
    first_sum = false;
  }
  CHD_CHECK(have0 || !first_sum, kErrInvalidArg, "Hoist: empty plan");
  // EvaluateFinalModDown, Hoist.cu:460-488
  const double in_scale = in.scale;
  const int in_slots = in.num_slots;
  CHD_TRY(res.reserve(P->level_np(level - 1), false, n));
  const uint32_t *src[2] = {fb, fa};
  uint32_t *dst[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, MDType::kModDownRescale, src, dst, 2));
  res.scale = pl.pt_scale * in_scale / P->rescale_prod[level];
  res.num_slots = std::max(in_slots, pl.pt_slots);
  return check_cuda("linear transform");
}

Status Context::lt_evaluate_batch(int count, DeviceCt *const *res, const DeviceCt *const *in, const LTPlan &pl,
                                  const RotKeys &keys) {
  // HoistHandler::Evaluate (Hoist.cu:554-975) for `count` ciphertexts at one
  // level: per ciphertext the hoisted baby steps and the giant-step
  // plaintext accumulation; across the batch every giant step's ModDown,
  // ModUp and key product, and the final ModDownAndRescale, run as one
  // batched launch sequence.  Each ciphertext's result equals lt_evaluate's.
  const bool only_gs = pl.bs_idx.size() == 1 && pl.bs_idx[0] == 0;
  if (only_gs) {
    for (int c = 0; c < count; c++) CHD_TRY(lt_evaluate(*res[c], *in[c], pl, keys));
    return kOk;
  }
  const int level = pl.pt_level;
  const int n = P->n;
  for (int c = 0; c < count; c++) {
    CHD_CHECK(!in[c]->has_rx && in[c]->np.aux == 0, kErrShape, "Hoist: input should be relinearized and mod-down");
    CHD_CHECK(in[c]->np == P->level_np(level), kErrShape, "Hoist: input level mismatch");
    for (int d = 0; d < count; d++)
      CHD_CHECK(c == d || res[c] != in[d], kErrInvalidArg, "Hoist: a result aliases another input of the batch");
  }
  const HoistOps H(*this, level);
  const size_t tw_ = H.tw;
  const NP qp = H.qp;
  auto key_of = [&](int r) -> const DeviceEvk * {
    auto it = keys.find(r);
    return it == keys.end() ? nullptr : it->second;
  };
  ArenaScope scope(arena);
  auto alloc = [&](size_t words) { return static_cast<uint32_t *>(arena.alloc(words * 4)); };
  // per ciphertext, for the whole call: ModUp digits, the final accumulator,
  // scratch of the giant steps and the giant-step sums
  std::vector<std::vector<uint32_t *>> mu(count, std::vector<uint32_t *>(H.m.beta));
  std::vector<uint32_t *const *> mu_p(count);
  std::vector<uint32_t *> fb(count), fa(count), md(count), tb(count), ta(count);
  std::vector<std::vector<std::pair<uint32_t *, uint32_t *>>> outs(count);
  std::map<int, int> slot_of, gpos;
  for (size_t i = 0; i < pl.bs_idx.size(); i++) slot_of[pl.bs_idx[i]] = static_cast<int>(i);
  for (size_t i = 0; i < pl.gs_idx.size(); i++) gpos[pl.gs_idx[i]] = static_cast<int>(i);
  std::vector<std::vector<std::pair<int, const uint32_t *>>> terms(pl.gs_idx.size());
  for (const auto &pt : pl.pts) terms[gpos[pt.gs]].push_back({slot_of[pt.bs], pt.dev});
  bool have0 = false;
  for (int x : pl.gs_idx) have0 = have0 || x == 0;
  for (int c = 0; c < count; c++) {
    for (int i = 0; i < H.m.beta; i++) {
      mu[c][i] = alloc(tw_);
      CHD_CHECK(mu[c][i], kErrAlloc, "Hoist: scratch allocation failed");
    }
    mu_p[c] = mu[c].data();
    fb[c] = alloc(tw_);
    fa[c] = alloc(tw_);
    md[c] = alloc(static_cast<size_t>(H.nq) * n);
    tb[c] = alloc(tw_);
    ta[c] = alloc(tw_);
    CHD_CHECK(fb[c] && fa[c] && md[c] && tb[c] && ta[c], kErrAlloc, "Hoist: scratch allocation failed");
    outs[c].resize(pl.gs_idx.size());
    for (size_t i = 0; i < pl.gs_idx.size(); i++) {
      if (pl.gs_idx[i] == 0) {
        outs[c][i] = {fb[c], fa[c]};
      } else {
        uint32_t *b = alloc(tw_), *a = alloc(tw_);
        CHD_CHECK(b && a, kErrAlloc, "Hoist: scratch allocation failed");
        outs[c][i] = {b, a};
      }
    }
  }
  // baby steps of every ciphertext (Hoist.cu:578-691): one batched ModUp
  // and one hoisted-rotation launch per kMaxHoistCts ciphertexts
  ArenaScope bs_scope(arena);  // released after the accumulation below
  std::vector<std::vector<DeviceCt>> bs(count);
  for (auto &v : bs) v.resize(pl.bs_idx.size());
  std::vector<int> rot_d;
  std::vector<const DeviceEvk *> rot_k;
  std::vector<size_t> rot_slot;
  for (size_t i = 0; i < pl.bs_idx.size(); i++) {
    const int r = pl.bs_idx[i];
    if (r == 0) continue;
    const DeviceEvk *k = key_of(r);
    CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(r));
    rot_d.push_back(r);
    rot_k.push_back(k);
    rot_slot.push_back(i);
  }
  std::vector<std::vector<DeviceCt *>> rot_o(count);
  std::vector<DeviceCt *const *> rot_op(count);
  std::vector<HoistOps::Pairs> ins(count, HoistOps::Pairs(pl.bs_idx.size()));
  for (int c = 0; c < count; c++) {
    for (size_t i = 0; i < pl.bs_idx.size(); i++) {
      if (pl.bs_idx[i] != 0) {
        CHD_TRY(scratch_ct(arena, bs[c][i], qp, false, n));
        ins[c][i] = {bs[c][i].bx, bs[c][i].ax};
      } else {
        uint32_t *b0 = alloc(tw_), *a0 = alloc(tw_);
        CHD_CHECK(b0 && a0, kErrAlloc, "Hoist: scratch allocation failed");
        H.pseudo_modup(in[c]->bx, b0);
        H.pseudo_modup(in[c]->ax, a0);
        ins[c][i] = {b0, a0};
      }
    }
    for (size_t s = 0; s < rot_slot.size(); s++) rot_o[c].push_back(&bs[c][rot_slot[s]]);
    rot_op[c] = rot_o[c].data();
  }
  if (!rot_d.empty())
    CHD_TRY(hoisted_rotate_batch(count, in, static_cast<int>(rot_d.size()), rot_d.data(), rot_k.data(),
                                 rot_op.data()));
  // giant-step plaintext accumulation (GSFusedPAccum, Hoist.cu:329-420), the
  // plaintexts read once per kMaxPtAccumCts ciphertexts
  CHD_TRY(H.pt_accum(count, ins, terms, outs));
  if (!have0) {
    // no giant step 0: the accumulator starts from zero
    for (int c = 0; c < count; c++) {
      cudaMemsetAsync(fb[c], 0, tw_ * 4, stream);
      cudaMemsetAsync(fa[c], 0, tw_ * 4, stream);
    }
  }
  // giant-step rotations (EvaluateGiantStepOptimized, Hoist.cu:860-975),
  // each step batched over the ciphertexts
  std::vector<const uint32_t *> src(count);
  for (size_t i = 0; i < pl.gs_idx.size(); i++) {
    const int gsr = pl.gs_idx[i];
    if (gsr == 0) continue;
    const DeviceEvk *k = key_of(gsr);
    CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(gsr));
    for (int c = 0; c < count; c++) src[c] = outs[c][i].second;
    CHD_TRY(moddown(level, MDType::kModDown, src.data(), md.data(), count));
    if (P->log_n == 16) {
      // ModUp and key product fused: the ModUp NTT rows feed the inner
      // product without a round trip through HBM
      std::vector<KSIn> ks(count);
      for (int c = 0; c < count; c++) ks[c] = KSIn{1, nullptr, md[c], nullptr, nullptr, tb[c], ta[c]};
      CHD_TRY(key_switch_fused(level, count, ks.data(), *k, MDType::kModDown, true));
    } else {
      CHD_TRY(modup_many(level, count, md.data(), mu_p.data()));
      CHD_TRY(H.key_mult(count, mu_p.data(), *k, tb.data(), ta.data()));
    }
    // key-switched part plus the accumulator's own b, both rotated, for
    // every ciphertext in few launches
    std::vector<const uint32_t *> ps(2 * count), ps2(2 * count);
    std::vector<uint32_t *> pd(2 * count);
    for (int c = 0; c < count; c++) {
      ps[2 * c] = tb[c];
      ps2[2 * c] = outs[c][i].first;
      pd[2 * c] = fb[c];
      ps[2 * c + 1] = ta[c];
      ps2[2 * c + 1] = nullptr;
      pd[2 * c + 1] = fa[c];
    }
    H.permute_add_many(2 * count, ps.data(), ps2.data(), pd.data(), gsr);
  }
  // EvaluateFinalModDown, Hoist.cu:460-488, all ciphertexts at once
  std::vector<const uint32_t *> fsrc(2 * count);
  std::vector<uint32_t *> fdst(2 * count);
  std::vector<double> in_scale(count);
  std::vector<int> in_slots(count);
  for (int c = 0; c < count; c++) {
    in_scale[c] = in[c]->scale;
    in_slots[c] = in[c]->num_slots;
  }
  for (int c = 0; c < count; c++) {
    CHD_TRY(res[c]->reserve(P->level_np(level - 1), false, n));
    fsrc[2 * c] = fb[c];
    fsrc[2 * c + 1] = fa[c];
    fdst[2 * c] = res[c]->bx;
    fdst[2 * c + 1] = res[c]->ax;
  }
  CHD_TRY(moddown(level, MDType::kModDownRescale, fsrc.data(), fdst.data(), 2 * count));
  for (int c = 0; c < count; c++) {
    res[c]->scale = pl.pt_scale * in_scale[c] / P->rescale_prod[level];
    res[c]->num_slots = std::max(in_slots[c], pl.pt_slots);
  }
  return check_cuda("linear transform");
}

}  // namespace chd
