// The remaining public operations of the reference Context
// (src/core/Context.cpp), on the library's kernels:
//   Copy (:132-143), MultUnsafe Ct x Ct and Ct x Const at a target level
//   (:357-500, reading past the inputs' extra terminal primes), MadUnsafe
//   (:873-915), Permute / PermuteConjugate (:502-547), HConjAdd (:836-860),
//   LevelDown (:917-929), MultKeyNoModDown (:650-700), Add / Sub with a
//   plaintext (:171-186, :231-246), Sub of a constant (:248-263), the
//   reversed Sub(Pt, Ct) / Sub(Const, Ct) (:265-304) and MultUnsafe Ct x Pt
//   (:414-456);
//   IsMultUnsafeCompatible (:357-368) is in evalmod.cu.
#include <cmath>

#include "host.h"
#include "kernels.h"

namespace chd {
namespace {

uint32_t *part_ptr(DeviceCt &c, int p) { return p == 0 ? c.bx : (p == 1 ? c.ax : c.rx); }
const uint32_t *part_ptr(const DeviceCt &c, int p) { return p == 0 ? c.bx : (p == 1 ? c.ax : c.rx); }

struct CTerm {
  const DeviceCt *src;
  int front;           // rows of src skipped at the front (extra terminal primes)
  const uint32_t *c;   // per destination row Montgomery constant
};

// dst parts (over np's q rows) = sum_t src_t (.) c_t
void caccum(Context &C, DeviceCt &dst, const NP &np, int parts, const std::vector<CTerm> &terms) {
  const int nq = np.q(), n = C.P->n;
  std::vector<int> g(nq);
  C.P->gidx(np, g.data());
  ConstAccumDesc d{};
  for (const CTerm &t : terms) {
    for (int p = 0; p < parts; p++) d.src[d.terms][p] = part_ptr(*t.src, p);
    d.src_row0[d.terms] = t.front;
    for (int r = 0; r < nq; r++) d.c[d.terms][r] = t.c[r];
    d.terms++;
  }
  for (int p = 0; p < parts; p++) d.dst[p] = part_ptr(dst, p);
  for (int r = 0; r < nq; r++) {
    d.q[r] = C.P->primes[g[r]];
    d.qinv[r] = C.P->qinv[g[r]];
  }
  d.rows = nq;
  d.parts = parts;
  d.n = n;
  launch_const_accum(d, C.stream);
}

bool subset(const NP &sub, const NP &sup) { return sub.main <= sup.main && sub.ter <= sup.ter; }

// Context.cpp:54-60 (AssertSameScale)
bool same_scale(double s1, double s2) { return std::fabs(s1 - s2) < 1e-12 * s1; }

}  // namespace

Status Context::copy_ct(DeviceCt &res, const DeviceCt &a) {
  if (&res == &a) return kOk;
  const NP np = a.np;
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, rx, P->n));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 4;
  for (int p = 0; p < (rx ? 3 : 2); p++)
    cudaMemcpyAsync(part_ptr(res, p), part_ptr(a, p), bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return check_cuda("copy");
}

Status Context::mult_unsafe(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, int level) {
  CHD_CHECK(!a.has_rx && !b.has_rx, kErrShape, "Relinearization required before MultUnsafe Ct x Ct");
  CHD_CHECK(a.np.aux == 0 && b.np.aux == 0, kErrShape,
            "MultUnsafe Ct x Ct should be only used for ciphertexts without aux primes");
  const int la = P->np_to_level(a.np), lb = P->np_to_level(b.np);
  CHD_CHECK(la >= 0 && lb >= 0, kErrInvalidLevel, "MultUnsafe: invalid input level");
  if (level == -1) level = std::min(la, lb);
  CHD_CHECK(level >= 0 && level <= P->max_level, kErrInvalidLevel, "MultUnsafe: invalid target level");
  const NP np = P->level_np(level);
  CHD_CHECK(subset(np, a.np) && subset(np, b.np), kErrShape, "Incompatible levels for MultUnsafe Ct x Ct");
  if (&res == &a || &res == &b) {
    DeviceCt tmp;
    CHD_TRY(mult_unsafe(tmp, a, b, level));
    res = std::move(tmp);
    return kOk;
  }
  const int fa = a.np.ter - np.ter, fb = b.np.ter - np.ter, nq = np.q(), n = P->n;
  CHD_TRY(res.reserve(np, true, n));
  std::vector<int> g(nq);
  P->gidx(np, g.data());
  TensorBatch tb{};
  for (int r = 0; r < nq; r++) {
    if (tb.count == 64) {
      launch_tensor(tb, P->log_n, stream);
      tb.count = 0;
    }
    TensorRow &row = tb.rows[tb.count++];
    const size_t oa = static_cast<size_t>(fa + r) * n, ob = static_cast<size_t>(fb + r) * n;
    row.b1 = a.bx + oa;
    row.a1 = a.ax + oa;
    row.b2 = b.bx + ob;
    row.a2 = b.ax + ob;
    row.d0 = res.bx + static_cast<size_t>(r) * n;
    row.d1 = res.ax + static_cast<size_t>(r) * n;
    row.d2 = res.rx + static_cast<size_t>(r) * n;
    row.q = P->primes[g[r]];
    row.qinv = P->qinv[g[r]];
  }
  launch_tensor(tb, P->log_n, stream);
  res.scale = a.scale * b.scale;
  res.num_slots = std::max(a.num_slots, b.num_slots);
  return check_cuda("mult unsafe");
}

Status Context::mult_unsafe_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, int const_level,
                                  double const_scale, int level) {
  const int la = P->np_to_level(NP{a.np.main, a.np.ter, 0});
  CHD_CHECK(la >= 0, kErrInvalidLevel, "MultUnsafe: invalid input level");
  CHD_CHECK(const_level >= 0 && const_level <= P->max_level, kErrInvalidLevel, "MultUnsafe: invalid constant level");
  if (level == -1) level = std::min(la, const_level);
  CHD_CHECK(level >= 0 && level <= P->max_level, kErrInvalidLevel, "MultUnsafe: invalid target level");
  const NP np = P->level_np(level), cnp = P->level_np(const_level);
  CHD_CHECK(subset(np, a.np) && subset(np, cnp), kErrShape, "Incompatible levels for MultUnsafe Ct x Const");
  if (&res == &a && la != level) {
    DeviceCt tmp;
    CHD_TRY(mult_unsafe_const(tmp, a, cx, const_level, const_scale, level));
    res = std::move(tmp);
    return kOk;
  }
  const bool rx = a.has_rx;
  const double sc = a.scale * const_scale;
  const int slots = a.num_slots;
  const int fa = a.np.ter - np.ter;
  CHD_TRY(res.reserve(np, rx, P->n));
  caccum(*this, res, np, rx ? 3 : 2, {{&a, fa, cx + (cnp.ter - np.ter)}});
  res.scale = sc;
  res.num_slots = slots;
  return check_cuda("mult unsafe const");
}

Status Context::mad_unsafe(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, int const_level,
                           double const_scale) {
  CHD_CHECK(res.np.aux == 0 && a.np.aux == 0, kErrShape, "MadUnsafe should be only used for q primes");
  CHD_CHECK(const_level >= 0 && const_level <= P->max_level, kErrInvalidLevel, "MadUnsafe: invalid constant level");
  const NP np = res.np, cnp = P->level_np(const_level);
  CHD_CHECK(np.q() > 0 && subset(np, a.np) && subset(np, cnp), kErrShape, "Incompatible levels for MultUnsafe Ct x Const");
  CHD_CHECK(res.num_slots == a.num_slots, kErrInvalidArg, "MadUnsafe should be only used for the same number of slots");
  const double want = a.scale * const_scale;
  CHD_CHECK(std::fabs(res.scale - want) <= 1e-9 * std::fabs(want), kErrInvalidArg, "MadUnsafe: scale mismatch");
  CHD_CHECK(&res != &a, kErrInvalidArg, "MadUnsafe does not support res aliasing a");
  const int n = P->n;
  if (a.has_rx && !res.has_rx) {
    // res gains a zero third part (PrepareRx), then accumulates a's; its
    // two parts move to buffers with room for the third one when needed
    const size_t bytes = static_cast<size_t>(np.total()) * n * 4;
    if (!res.rx) {
      DeviceCt grown;
      CHD_TRY(grown.reserve(np, true, n));
      cudaMemcpyAsync(grown.bx, res.bx, bytes, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(grown.ax, res.ax, bytes, cudaMemcpyDeviceToDevice, stream);
      grown.scale = res.scale;
      grown.num_slots = res.num_slots;
      res = std::move(grown);
    }
    cudaMemsetAsync(res.rx, 0, bytes, stream);
    res.np = np;
    res.has_rx = true;
  }
  std::vector<uint32_t> one(np.q());
  std::vector<int> g(np.q());
  P->gidx(np, g.data());
  for (int r = 0; r < np.q(); r++) one[r] = prime::to_mont(1, P->primes[g[r]]);
  // res = a (.) c + res (.) 1 over the parts of a (res's own third part
  // stays when a has none)
  caccum(*this, res, np, a.has_rx ? 3 : 2,
         {{&a, a.np.ter - np.ter, cx + (cnp.ter - np.ter)}, {&res, 0, one.data()}});
  return check_cuda("mad unsafe");
}

Status Context::permute_ct(DeviceCt &res, const DeviceCt &a, int rot_dist, bool conjugate) {
  int amount = -1;
  if (!conjugate) {
    const int slots = a.num_slots > 0 ? a.num_slots : P->n / 2;
    amount = rot_dist % slots;
    if (amount < 0) amount += slots;
    if (amount == 0) return copy_ct(res, a);
  }
  if (&res == &a) {
    DeviceCt tmp;
    CHD_TRY(permute(tmp, a, amount));
    res = std::move(tmp);
    return kOk;
  }
  return permute(res, a, amount);
}

Status Context::hconj_add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key) {
  CHD_CHECK(a.np == b.np, kErrShape, "HConjAdd: level mismatch");
  ArenaScope scope(arena);
  DeviceCt tmp;
  CHD_TRY(scratch_ct(arena, tmp, a.np, false, P->n));
  CHD_TRY(hconj(tmp, a, key));
  return add(res, tmp, b);
}

Status Context::level_down(DeviceCt &res, const DeviceCt &a, int target_level) {
  CHD_CHECK(a.np.aux == 0, kErrShape, "LevelDown: ciphertext must not carry aux primes");
  const int level = P->np_to_level(a.np);
  CHD_CHECK(level >= 0 && target_level >= 0 && level >= target_level, kErrInvalidLevel,
            "Invalid target level for LevelDown");
  // the level-down constants are those of levels 1 .. default encryption
  // level (Context.cpp:102-107)
  CHD_CHECK(level <= P->spec.default_encryption_level, kErrInvalidLevel,
            "LevelDown: input above the default encryption level (no level-down constant there)");
  if (level == target_level) return copy_ct(res, a);
  // per level: times the constant 1 at that level's scale, then Rescale
  DeviceCt cur, tmp;
  const DeviceCt *prev = &a;
  std::vector<uint32_t> cx;
  for (int i = level; i > target_level; i--) {
    encode_const(i, P->scale.at(i), 1.0, 0, &cx);
    CHD_TRY(mult_const(tmp, *prev, cx.data(), P->scale.at(i)));
    CHD_TRY(rescale(cur, tmp));
    prev = &cur;
  }
  if (&res == &a) {
    res = std::move(cur);
    return kOk;
  }
  return copy_ct(res, cur);
}

Status Context::mult_key_no_moddown(DeviceCt &accum, const DeviceCt &a, const DeviceEvk &key) {
  CHD_CHECK(a.np.aux == 0, kErrShape, "MultKeyNoModDown is not supported for ciphertexts with p primes");
  CHD_CHECK(&accum != &a, kErrInvalidArg, "In-place operation is not supported for MultKeyNoModDown");
  const int level = P->np_to_level(a.np);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "MultKeyNoModDown: invalid level");
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(accum.reserve(P->level_np(level, P->alpha), false, P->n));
  // with rx: ModUp(rx) (.) key + P * (bx, ax) (relinearisation); without:
  // ModUp(ax) (.) key + (P * bx, 0) (the key switch of a rotation)
  if (a.has_rx)
    CHD_TRY(key_switch_core(level, a.bx, a.ax, a.rx, key, accum.bx, accum.ax));
  else
    CHD_TRY(key_switch_core(level, a.bx, nullptr, a.ax, key, accum.bx, accum.ax));
  accum.scale = sc;
  accum.num_slots = slots;
  return check_cuda("mult key no moddown");
}

// res.bx = a.bx (+/-) pt, ax and rx copied (Context.cpp:171-186, 231-246)
Status Context::add_sub_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt, double pscale, bool subtract) {
  CHD_CHECK(same_scale(a.scale, pscale), kErrInvalidArg, "Scale mismatch");
  const NP np = a.np;
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  const uint32_t *pa[1] = {a.bx}, *pb[1] = {pt};
  const uint32_t *keep[2] = {a.ax, a.rx};
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[1] = {res.bx};
  CHD_TRY(elem_parts(*this, subtract ? ElemOp::kSub : ElemOp::kAdd, np, 1, pd, pa, pb, nullptr));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 4;
  if (keep[0] != res.ax) cudaMemcpyAsync(res.ax, keep[0], bytes, cudaMemcpyDeviceToDevice, stream);
  if (rx && keep[1] != res.rx) cudaMemcpyAsync(res.rx, keep[1], bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return check_cuda("add / sub plain");
}

// res.bx = a.bx - c, ax and rx copied (Context.cpp:248-263)
Status Context::sub_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx) {
  const NP np = a.np;
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  const uint32_t *pa[1] = {a.bx};
  const uint32_t *keep[2] = {a.ax, a.rx};
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[1] = {res.bx};
  CHD_TRY(elem_parts(*this, ElemOp::kSubConst, np, 1, pd, pa, nullptr, cx));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 4;
  if (keep[0] != res.ax) cudaMemcpyAsync(res.ax, keep[0], bytes, cudaMemcpyDeviceToDevice, stream);
  if (rx && keep[1] != res.rx) cudaMemcpyAsync(res.rx, keep[1], bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return check_cuda("sub const");
}

// res = pt - b or c - b: bx = pt - b.bx (c - b.bx), ax = -b.ax, rx = -b.rx
// (Context.cpp:265-304); exactly one of pt / cx is given
Status Context::sub_from(DeviceCt &res, const uint32_t *pt, const uint32_t *cx, double scale, const DeviceCt &b) {
  CHD_CHECK((pt != nullptr) != (cx != nullptr), kErrInvalidArg, "Sub: give a plaintext or a constant");
  CHD_CHECK(same_scale(scale, b.scale), kErrInvalidArg, "Scale mismatch");
  const NP np = b.np;
  const bool rx = b.has_rx;
  const int slots = b.num_slots;
  const uint32_t *pbx[1] = {b.bx}, *ppt[1] = {pt};
  const uint32_t *prest[2] = {b.ax, b.rx};
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[1] = {res.bx};
  if (pt)
    CHD_TRY(elem_parts(*this, ElemOp::kSub, np, 1, pd, ppt, pbx, nullptr));
  else
    CHD_TRY(elem_parts(*this, ElemOp::kSubOppConst, np, 1, pd, pbx, nullptr, cx));
  uint32_t *prd[2] = {res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kNeg, np, rx ? 2 : 1, prd, prest, nullptr, nullptr));
  res.scale = scale;
  res.num_slots = slots;
  return check_cuda("sub from");
}

// Context.cpp:414-456: res = a (.) pt at `level` (-1: the lower level), both
// read past their extra terminal primes; aux primes: the fewer of the two
Status Context::mult_unsafe_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt, int pt_level, int pt_aux,
                                  double pscale, int level) {
  const int la = P->np_to_level(NP{a.np.main, a.np.ter, 0});
  CHD_CHECK(la >= 0, kErrInvalidLevel, "MultUnsafe: invalid input level");
  CHD_CHECK(pt_level >= 0 && pt_level <= P->max_level, kErrInvalidLevel, "MultUnsafe: invalid plaintext level");
  CHD_CHECK(pt_aux >= 0 && pt_aux <= P->alpha, kErrShape, "MultUnsafe: invalid plaintext aux prime count");
  if (level == -1) level = std::min(la, pt_level);
  CHD_CHECK(level >= 0 && level <= P->max_level, kErrInvalidLevel, "MultUnsafe: invalid target level");
  const int aux = std::min(a.np.aux, pt_aux);
  const NP np = P->level_np(level, aux), pnp = P->level_np(pt_level, pt_aux);
  CHD_CHECK(subset(np, a.np) && subset(np, pnp), kErrShape, "Incompatible levels for MultUnsafe Ct x Pt");
  if (&res == &a && la != level) {
    DeviceCt tmp;
    CHD_TRY(mult_unsafe_plain(tmp, a, pt, pt_level, pt_aux, pscale, level));
    res = std::move(tmp);
    return kOk;
  }
  const bool rx = a.has_rx;
  const double sc = a.scale * pscale;
  const int slots = a.num_slots;
  const size_t n = P->n, fa = (a.np.ter - np.ter) * n, fp = (pnp.ter - np.ter) * n;
  const uint32_t *pa[3] = {a.bx + fa, a.ax + fa, rx ? a.rx + fa : nullptr};
  const uint32_t *pp[3] = {pt + fp, pt + fp, pt + fp};
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kMult, np, rx ? 3 : 2, pd, pa, pp, nullptr));
  res.scale = sc;
  res.num_slots = slots;
  return check_cuda("mult unsafe plain");
}

}  // namespace chd
