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
  // HoistHandler::EvaluateMinKSBabyStep / EvaluateMinKSGiantStep
  // (Hoist.cu:490-552): baby steps by repeated HRot with the baby stride,
  // giant steps in reverse order, accumulate, HRot by the giant stride,
  // then Rescale.  Works in the Q basis of pt_level.
  const int level = pl.pt_level;
  const int n = P->n;
  CHD_CHECK(!in.has_rx && in.np.aux == 0, kErrShape, "Hoist: input should be relinearized and mod-down");
  CHD_CHECK(in.np == P->level_np(level), kErrShape, "Hoist: input level mismatch");
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
  std::vector<int> g(nq);
  P->gidx(np, g.data());
  ArenaScope scope(arena);
  // baby steps in the Q basis
  std::vector<DeviceCt> bs(pl.bs_idx.size());
  std::map<int, int> slot_of;
  for (size_t i = 0; i < pl.bs_idx.size(); i++) {
    CHD_TRY(scratch_ct(arena, bs[i], np, false, n));
    slot_of[pl.bs_idx[i]] = static_cast<int>(i);
  }
  const DeviceEvk *kb = key_of(bs_stride);
  for (size_t i = 0; i < pl.bs_idx.size(); i++) {
    const int r = pl.bs_idx[i];
    if (r == 0) {
      const size_t bytes = static_cast<size_t>(nq) * n * 4;
      cudaMemcpyAsync(bs[i].bx, in.bx, bytes, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(bs[i].ax, in.ax, bytes, cudaMemcpyDeviceToDevice, stream);
      bs[i].scale = in.scale;
      bs[i].num_slots = in.num_slots;
    } else {
      CHD_CHECK(kb, kErrKey, "Hoist: missing rotation key " + std::to_string(bs_stride));
      auto it = slot_of.find(r - bs_stride);
      CHD_CHECK(it != slot_of.end(), kErrInvalidArg, "Hoist: MinKS baby-step sequence is not complete");
      CHD_TRY(hrot(bs[i], bs[it->second], *kb, bs_stride));
    }
  }
  // giant steps, reversed
  DeviceCt acc, tmp;
  CHD_TRY(scratch_ct(arena, acc, np, false, n));
  CHD_TRY(scratch_ct(arena, tmp, np, false, n));
  const DeviceEvk *kg = key_of(gs_stride);
  bool first = true;
  int prev = 0;
  for (auto git = pl.gs_idx.rbegin(); git != pl.gs_idx.rend(); ++git) {
    const int gsi = *git;
    PtAccumDesc d{};
    int nin = 0;
    std::map<int, int> in_of;
    PtAccumOut &po = d.out[0];
    for (const auto &pt : pl.pts) {
      if (pt.gs != gsi) continue;
      auto f = in_of.find(pt.bs);
      if (f == in_of.end()) {
        CHD_CHECK(nin < kMaxPtAccumIn, kErrUnsupported, "Hoist: too many baby steps");
        const DeviceCt &b = bs[slot_of.at(pt.bs)];
        d.in_b[nin] = b.bx;
        d.in_a[nin] = b.ax;
        f = in_of.emplace(pt.bs, nin++).first;
      }
      CHD_CHECK(po.terms < kMaxPtAccumTerms, kErrUnsupported, "Hoist: too many terms");
      po.term[po.terms] = static_cast<int16_t>(f->second);
      po.pt[po.terms] = pt.dev;  // the first nq rows are the q primes
      po.terms++;
    }
    for (int r = 0; r < nq; r++) {
      d.q[r] = P->primes[g[r]];
      d.qinv[r] = P->qinv[g[r]];
    }
    d.rows = nq;
    d.n = n;
    d.outs = 1;
    if (first) {
      po.b = acc.bx;
      po.a = acc.ax;
      launch_pt_accum(d, stream);
    } else {
      CHD_CHECK(prev == gsi + gs_stride, kErrInvalidArg, "Hoist: MinKS giant-step sequence is not complete");
      po.b = tmp.bx;
      po.a = tmp.ax;
      launch_pt_accum(d, stream);
      CHD_TRY(add(acc, acc, tmp));
    }
    acc.scale = in.scale * pl.pt_scale;
    acc.num_slots = std::max(in.num_slots, pl.pt_slots);
    if (gsi != 0) {
      CHD_CHECK(kg, kErrKey, "Hoist: missing rotation key " + std::to_string(gs_stride));
      CHD_TRY(hrot(tmp, acc, *kg, gs_stride));
      const size_t bytes = static_cast<size_t>(nq) * n * 4;
      cudaMemcpyAsync(acc.bx, tmp.bx, bytes, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(acc.ax, tmp.ax, bytes, cudaMemcpyDeviceToDevice, stream);
    } else {
      CHD_CHECK(first || prev == gs_stride, kErrInvalidArg, "Hoist: MinKS giant-step sequence is not complete");
    }
    first = false;
    prev = gsi;
  }
  const double sc = acc.scale;
  CHD_TRY(rescale(res, acc));
  res.scale = sc / P->rescale_prod[level];
  return check_cuda("linear transform (min-KS)");
}

Status Context::lt_evaluate(DeviceCt &res, const DeviceCt &in, const LTPlan &pl, const RotKeys &keys) {
  // HoistHandler::Evaluate, Hoist.cu:554-975 (non-min-KS, fused kernels)
  const int level = pl.pt_level;
  const int n = P->n;
  CHD_CHECK(!in.has_rx && in.np.aux == 0, kErrShape, "Hoist: input should be relinearized and mod-down");
  CHD_CHECK(in.np == P->level_np(level), kErrShape, "Hoist: input level mismatch");
  const NP qp = P->level_np(level, P->alpha);
  const int nq = qp.q(), tot = qp.total();
  const LevelMS &m = lms(level);
  std::vector<int> g(tot);
  P->gidx(qp, g.data());
  const int prime_offset = P->max_ter - qp.ter;
  const size_t tw_ = static_cast<size_t>(tot) * n;
  auto key_of = [&](int r) -> const DeviceEvk * {
    auto it = keys.find(r);
    return it == keys.end() ? nullptr : it->second;
  };
  ArenaScope scope(arena);
  auto alloc = [&](size_t words) { return static_cast<uint32_t *>(arena.alloc(words * 4)); };
  // P * x on q rows, zero on aux rows (PseudoModUp + ZeroExtend)
  auto pseudo_modup = [&](const uint32_t *src, uint32_t *dst) {
    ConstAccumDesc d{};
    d.terms = 1;
    d.src[0][0] = src;
    d.src_row0[0] = 0;
    d.dst[0] = dst;
    for (int r = 0; r < nq; r++) {
      d.q[r] = P->primes[g[r]];
      d.qinv[r] = P->qinv[g[r]];
      d.c[0][r] = p_prod[prime_offset + r];
    }
    d.rows = nq;
    d.parts = 1;
    d.n = n;
    launch_const_accum(d, stream);
    cudaMemsetAsync(dst + static_cast<size_t>(nq) * n, 0, static_cast<size_t>(tot - nq) * n * 4, stream);
  };
  // sum_i ModUp(x)_i (.) key_i over Q u P (MultKeyNoModDown, Context.cpp:610-648)
  auto key_mult = [&](uint32_t *const *mu, const DeviceEvk &k, uint32_t *ob, uint32_t *oa) -> Status {
    CHD_CHECK(k.np.aux == P->alpha && k.np.q() == P->L, kErrKey, "Hoist: key basis mismatch");
    KeyMacDesc d{};
    const size_t kstride = static_cast<size_t>(P->L + P->alpha) * n;
    int nb = 0;
    for (int i = 0; i < m.beta; i++) {
      if (m.dig_e[i] <= 0) continue;
      CHD_CHECK(i < k.beta, kErrKey, "Hoist: key has too few digits");
      d.kb[nb] = k.bx + i * kstride;
      d.ka[nb] = k.ax + i * kstride;
      d.ct[0].mu[nb] = mu[i];
      nb++;
    }
    d.beta = nb;
    d.rows = tot;
    d.nq = nq;
    d.count = 1;
    for (int r = 0; r < tot; r++) {
      d.q[r] = P->primes[g[r]];
      d.qinv[r] = P->qinv[g[r]];
      d.p_prod[r] = 0;
      d.key_row[r] = static_cast<int16_t>(r < nq ? prime_offset + r : P->L + (r - nq));
    }
    d.ct[0].d0 = d.ct[0].d1 = nullptr;
    d.ct[0].acc_b = ob;
    d.ct[0].acc_a = oa;
    launch_key_mac(d, P->log_n, stream);
    return kOk;
  };
  // dst (+)= Permute_g(src) over the Q u P rows of one part
  auto permute_rows = [&](const uint32_t *src, uint32_t *dst, const uint32_t *add, int amount) {
    PermuteBatch pb{};
    pb.galois = P->galois_of(amount);
    for (int r = 0; r < tot; r++) {
      if (pb.count == 64) {
        launch_permute(pb, P->log_n, stream);
        pb.count = 0;
      }
      PermuteRow &pr = pb.rows[pb.count++];
      pr.src = src + static_cast<size_t>(r) * n;
      pr.dst = dst + static_cast<size_t>(r) * n;
      pr.add = add ? add + static_cast<size_t>(r) * n : nullptr;
      pr.q = P->primes[g[r]];
    }
    launch_permute(pb, P->log_n, stream);
  };
  auto add_rows = [&](const uint32_t *a, const uint32_t *b, uint32_t *dst, int rows) {
    ElemBatch eb{};
    for (int r = 0; r < rows; r++) {
      if (eb.count == kMaxElemRows) {
        launch_elementwise(ElemOp::kAdd, eb, P->log_n, stream);
        eb.count = 0;
      }
      ElemRow &e = eb.rows[eb.count++];
      e.a = a + static_cast<size_t>(r) * n;
      e.b = b + static_cast<size_t>(r) * n;
      e.dst = dst + static_cast<size_t>(r) * n;
      e.q = P->primes[g[r]];
      e.qinv = P->qinv[g[r]];
    }
    launch_elementwise(ElemOp::kAdd, eb, P->log_n, stream);
  };
  auto pt_accum = [&](const std::vector<std::pair<const uint32_t *, const uint32_t *>> &ins,
                      const std::vector<std::vector<std::pair<int, const uint32_t *>>> &terms,
                      const std::vector<std::pair<uint32_t *, uint32_t *>> &outs) -> Status {
    CHD_CHECK(static_cast<int>(ins.size()) <= kMaxPtAccumIn, kErrUnsupported, "Hoist: too many baby steps");
    for (size_t o0 = 0; o0 < outs.size(); o0 += kMaxPtAccumOuts) {
      PtAccumDesc d{};
      for (size_t i = 0; i < ins.size(); i++) {
        d.in_b[i] = ins[i].first;
        d.in_a[i] = ins[i].second;
      }
      for (int r = 0; r < tot; r++) {
        d.q[r] = P->primes[g[r]];
        d.qinv[r] = P->qinv[g[r]];
      }
      d.rows = tot;
      d.n = n;
      d.outs = static_cast<int>(std::min<size_t>(kMaxPtAccumOuts, outs.size() - o0));
      for (int o = 0; o < d.outs; o++) {
        const auto &t = terms[o0 + o];
        CHD_CHECK(static_cast<int>(t.size()) <= kMaxPtAccumTerms, kErrUnsupported, "Hoist: too many terms");
        PtAccumOut &po = d.out[o];
        po.b = outs[o0 + o].first;
        po.a = outs[o0 + o].second;
        po.terms = static_cast<int>(t.size());
        for (size_t k = 0; k < t.size(); k++) {
          po.term[k] = static_cast<int16_t>(t[k].first);
          po.pt[k] = t[k].second;
        }
      }
      launch_pt_accum(d, stream);
    }
    return kOk;
  };

  std::vector<uint32_t *> mu(m.beta);
  for (int i = 0; i < m.beta; i++) {
    mu[i] = alloc(tw_);
    CHD_CHECK(mu[i], kErrAlloc, "Hoist: scratch allocation failed");
  }
  uint32_t *fb = alloc(tw_), *fa = alloc(tw_);  // final accumulator (Q u P)
  CHD_CHECK(fb && fa, kErrAlloc, "Hoist: scratch allocation failed");
  const bool only_gs = pl.bs_idx.size() == 1 && pl.bs_idx[0] == 0;
  if (only_gs) {
    // Hoist.cu:706-808: ModUp(a) once, per giant step key mult + P b, times pt,
    // then PermuteAccum
    CHD_TRY(modup(level, in.ax, mu.data()));
    uint32_t *bxp = alloc(tw_), *tb = alloc(tw_), *ta = alloc(tw_);
    uint32_t *p0b = alloc(tw_), *p0a = alloc(tw_);
    CHD_CHECK(bxp && tb && ta && p0b && p0a, kErrAlloc, "Hoist: scratch allocation failed");
    pseudo_modup(in.bx, bxp);
    bool have0 = false;
    bool first_sum = true;
    for (const auto &pt : pl.pts) {
      if (pt.gs == 0) {
        pseudo_modup(in.ax, p0a);
        CHD_TRY(pt_accum({{bxp, p0a}}, {{{0, pt.dev}}}, {{fb, fa}}));
        have0 = true;
      }
    }
    for (const auto &pt : pl.pts) {
      if (pt.gs == 0) continue;
      const DeviceEvk *k = key_of(pt.gs);
      CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(pt.gs));
      CHD_TRY(key_mult(mu.data(), *k, tb, ta));
      add_rows(tb, bxp, tb, nq);
      CHD_TRY(pt_accum({{tb, ta}}, {{{0, pt.dev}}}, {{p0b, p0a}}));
      if (!have0 && first_sum) {
        permute_rows(p0b, fb, nullptr, pt.gs);
        permute_rows(p0a, fa, nullptr, pt.gs);
      } else {
        permute_rows(p0b, fb, fb, pt.gs);
        permute_rows(p0a, fa, fa, pt.gs);
      }
      first_sum = false;
    }
    CHD_CHECK(have0 || !first_sum, kErrInvalidArg, "Hoist: empty plan");
  } else {
    // baby steps (Hoist.cu:578-691)
    std::vector<DeviceCt> bs(pl.bs_idx.size());
    for (size_t i = 0; i < pl.bs_idx.size(); i++)
      if (pl.bs_idx[i] != 0) CHD_TRY(scratch_ct(arena, bs[i], qp, false, n));
    std::vector<int> rot_d;
    std::vector<const DeviceEvk *> rot_k;
    std::vector<DeviceCt *> rot_o;
    std::map<int, int> slot_of;
    for (size_t i = 0; i < pl.bs_idx.size(); i++) {
      const int r = pl.bs_idx[i];
      slot_of[r] = static_cast<int>(i);
      if (r == 0) continue;
      const DeviceEvk *k = key_of(r);
      CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(r));
      rot_d.push_back(r);
      rot_k.push_back(k);
      rot_o.push_back(&bs[i]);
    }
    if (!rot_d.empty()) CHD_TRY(hoisted_rotate(in, static_cast<int>(rot_d.size()), rot_d.data(), rot_k.data(), rot_o.data()));
    std::vector<std::pair<const uint32_t *, const uint32_t *>> ins(pl.bs_idx.size());
    for (size_t i = 0; i < pl.bs_idx.size(); i++) {
      if (pl.bs_idx[i] == 0) {
        uint32_t *b0 = alloc(tw_), *a0 = alloc(tw_);
        CHD_CHECK(b0 && a0, kErrAlloc, "Hoist: scratch allocation failed");
        pseudo_modup(in.bx, b0);
        pseudo_modup(in.ax, a0);
        ins[i] = {b0, a0};
      } else {
        ins[i] = {bs[i].bx, bs[i].ax};
      }
    }
    // giant-step plaintext accumulation (GSFusedPAccum, Hoist.cu:329-420)
    std::vector<std::vector<std::pair<int, const uint32_t *>>> terms(pl.gs_idx.size());
    std::vector<std::pair<uint32_t *, uint32_t *>> outs(pl.gs_idx.size());
    std::map<int, int> gpos;
    for (size_t i = 0; i < pl.gs_idx.size(); i++) gpos[pl.gs_idx[i]] = static_cast<int>(i);
    for (const auto &pt : pl.pts) terms[gpos[pt.gs]].push_back({slot_of[pt.bs], pt.dev});
    bool have0 = false;
    for (size_t i = 0; i < pl.gs_idx.size(); i++) {
      if (pl.gs_idx[i] == 0) {
        outs[i] = {fb, fa};
        have0 = true;
      } else {
        uint32_t *b = alloc(tw_), *a = alloc(tw_);
        CHD_CHECK(b && a, kErrAlloc, "Hoist: scratch allocation failed");
        outs[i] = {b, a};
      }
    }
    CHD_TRY(pt_accum(ins, terms, outs));
    if (!have0) {
      // no giant step 0: the accumulator starts from zero
      cudaMemsetAsync(fb, 0, tw_ * 4, stream);
      cudaMemsetAsync(fa, 0, tw_ * 4, stream);
    }
    // giant-step rotations (EvaluateGiantStepOptimized, Hoist.cu:860-975)
    uint32_t *md = alloc(static_cast<size_t>(nq) * n), *tb = alloc(tw_), *ta = alloc(tw_);
    CHD_CHECK(md && tb && ta, kErrAlloc, "Hoist: scratch allocation failed");
    for (size_t i = 0; i < pl.gs_idx.size(); i++) {
      const int gsr = pl.gs_idx[i];
      if (gsr == 0) continue;
      const DeviceEvk *k = key_of(gsr);
      CHD_CHECK(k, kErrKey, "Hoist: missing rotation key " + std::to_string(gsr));
      const uint32_t *src[1] = {outs[i].second};
      uint32_t *dst[1] = {md};
      CHD_TRY(moddown(level, MDType::kModDown, src, dst, 1));
      CHD_TRY(modup(level, md, mu.data()));
      CHD_TRY(key_mult(mu.data(), *k, tb, ta));
      // key-switched part plus the accumulator's own b, both rotated
      add_rows(tb, outs[i].first, tb, tot);
      permute_rows(tb, fb, fb, gsr);
      permute_rows(ta, fa, fa, gsr);
    }
  }
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

}  // namespace chd
