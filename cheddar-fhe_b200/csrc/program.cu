// Device interpreter of op programs (compiled EvalPoly / EvalMod / Boot).
//
// Every op writes a spare ciphertext, which is then swapped into the
// destination register, so outputs may alias inputs freely.  The op
// semantics are the reference Context's (src/core/Context.cpp):
// MultUnsafe Ct x Const / Ct x Ct at a target level reading the inputs'
// limbs past their extra terminal primes ("front ignore"), CAccum,
// Add / Sub with mixed Rx, RelinearizeRescale, Rescale, LevelDown through
// the level-down constant, HConj, MultImaginaryUnit, ModUpToMax, HRotAdd
// and linear transforms.
#include <algorithm>

#include "host.h"
#include "kernels.h"

namespace chd {
namespace {

}  // namespace

void swap_regs(DeviceCt &x, DeviceCt &y) {
  std::swap(x.np, y.np);
  std::swap(x.has_rx, y.has_rx);
  std::swap(x.scale, y.scale);
  std::swap(x.num_slots, y.num_slots);
  std::swap(x.bx, y.bx);
  std::swap(x.ax, y.ax);
  std::swap(x.rx, y.rx);
  std::swap(x.cap_words, y.cap_words);
  std::swap(x.owned, y.owned);
}

namespace {

uint32_t *part_of(DeviceCt &c, int p) { return p == 0 ? c.bx : (p == 1 ? c.ax : c.rx); }
const uint32_t *part_of(const DeviceCt &c, int p) { return p == 0 ? c.bx : (p == 1 ? c.ax : c.rx); }

}  // namespace

Status Context::program_regs(const Program &prog, std::vector<DeviceCt> &regs) {
  // registers plus two spares, all at top-level capacity with an Rx part,
  // so that no op reallocates (a reallocation synchronises the device).
  // Registers that already have the capacity keep their contents.
  if (static_cast<int>(regs.size()) < prog.nregs + 2) regs.resize(prog.nregs + 2);
  const NP top = P->level_np(P->max_level);
  const size_t words = static_cast<size_t>(top.total()) * P->n;
  for (auto &r : regs) {
    if (r.cap_words < words || !r.rx) {
      CHD_CHECK(r.cap_words == 0, kErrInvalidArg, "program: register would lose its contents");
      CHD_TRY(r.reserve(top, true, P->n));
      r.np = NP{};
      r.has_rx = false;
    }
  }
  return kOk;
}

Status Context::run_program(const Program &prog, std::vector<DeviceCt> &regs, const ProgKeys &keys,
                            const std::vector<const LTPlan *> *lts) {
  std::vector<DeviceCt> *r = &regs;
  return run_program_batch(prog, 1, &r, keys, lts);
}

namespace {
// Per-ciphertext launches of one op on alternating streams: forks the
// context's second stream from the context stream at construction, selects
// the stream of ciphertext i, and at destruction (every exit path) restores
// the context stream and joins the second stream back into it.
struct Alternation {
  Context &C;
  bool on;
  cudaStream_t main;
  Alternation(Context &c, bool want) : C(c), on(want), main(c.stream) {
    if (on)
      on = cudaEventRecord(C.ev_fork, main) == cudaSuccess && cudaStreamWaitEvent(C.aux_stream, C.ev_fork, 0) == cudaSuccess;
  }
  void select(int i) {
    if (on) C.stream = (i & 1) ? C.aux_stream : main;
  }
  void finish() {
    if (!on) return;
    on = false;
    C.stream = main;
    if (cudaEventRecord(C.ev_join, C.aux_stream) == cudaSuccess) cudaStreamWaitEvent(main, C.ev_join, 0);
  }
  ~Alternation() { finish(); }
  Alternation(const Alternation &) = delete;
  Alternation &operator=(const Alternation &) = delete;
};
}  // namespace

Status Context::run_program_batch(const Program &prog, int count, std::vector<DeviceCt> *const *R,
                                  const ProgKeys &keys, const std::vector<const LTPlan *> *lts) {
  // The program on `count` ciphertexts, each with its own registers R[c]:
  // key switches (RelinearizeRescale, HConj, HRotAdd), rescales and linear
  // transforms run once over the whole batch (fused launches of all its
  // ciphertexts); the element-wise ops run per ciphertext.  Every
  // ciphertext's result equals a run of the program on it alone.
  const DeviceEvk *mult_key = keys.mult, *conj_key = keys.conj;
  const RotKeys *rot_keys = keys.rot;
  CHD_CHECK(count >= 1, kErrInvalidArg, "program: empty batch");
  for (int c = 0; c < count; c++) CHD_TRY(program_regs(prog, *R[c]));
  const int n = P->n;
  // constants: Montgomery residues over their own level's q primes
  std::vector<std::vector<uint32_t>> cx(prog.consts.size());
  std::vector<NP> cnp(prog.consts.size());
  for (size_t i = 0; i < prog.consts.size(); i++) {
    const ProgConst &c = prog.consts[i];
    encode_const(c.level, c.scale, c.value, 0, &cx[i]);
    cnp[i] = P->level_np(c.level);
  }
  // dst (parts) = sum over terms of src_t (.) c_t, at np, each term reading
  // its source from row `front_t`
  struct Term {
    const DeviceCt *src;
    int front;
    const uint32_t *c;  // per dst row constant (Montgomery), already offset
  };
  // One launch takes every part of the destination; while `defer` is set
  // (the per-ciphertext loop of one op over a batch), the accumulations of
  // consecutive ciphertexts, which share the op's constants, join one launch
  // until its outputs run out or the terms differ; flush_accum launches it.
  ConstAccumDesc pend{};
  const uint32_t *pend_c[kMaxConstAccumTerms] = {};
  bool defer = false;
  auto flush_accum = [&]() {
    if (pend.parts > 0) launch_const_accum(pend, stream);
    pend.parts = 0;
    pend.terms = 0;
  };
  auto const_accum = [&](DeviceCt &dst, const NP &np, int parts, const std::vector<Term> &terms) -> Status {
    const int nq = np.q();
    if (terms.empty()) {
      for (int p = 0; p < parts; p++) cudaMemsetAsync(part_of(dst, p), 0, static_cast<size_t>(nq) * n * 4, stream);
      return kOk;
    }
    CHD_CHECK(static_cast<int>(terms.size()) <= kMaxConstAccumTerms, kErrUnsupported,
              "program: too many accumulation terms");
    bool same = pend.parts > 0 && pend.rows == nq && pend.terms == static_cast<int>(terms.size()) &&
                pend.parts + parts <= kMaxConstAccumOuts;
    for (size_t i = 0; same && i < terms.size(); i++)
      same = pend_c[i] == terms[i].c && pend.src_row0[i] == terms[i].front;
    if (!same) {
      flush_accum();
      std::vector<int> g(nq);
      P->gidx(np, g.data());
      for (size_t i = 0; i < terms.size(); i++) {
        pend.src_row0[i] = terms[i].front;
        pend_c[i] = terms[i].c;
        for (int r = 0; r < nq; r++) pend.c[i][r] = terms[i].c[r];
      }
      for (int r = 0; r < nq; r++) {
        pend.q[r] = P->primes[g[r]];
        pend.qinv[r] = P->qinv[g[r]];
      }
      pend.terms = static_cast<int>(terms.size());
      pend.rows = nq;
      pend.n = n;
    }
    for (int p = 0; p < parts; p++) {
      const int o = pend.parts++;
      for (size_t i = 0; i < terms.size(); i++)
        pend.src[i][o] = (p == 2 && !terms[i].src->has_rx) ? nullptr : part_of(*terms[i].src, p);
      pend.dst[o] = part_of(dst, p);
    }
    if (!defer) flush_accum();
    return kOk;
  };
  auto front_of = [&](const NP &src, const NP &dst) -> int { return src.ter - dst.ter; };
  auto check_subset = [&](const NP &sub, const NP &sup) -> Status {
    CHD_CHECK(sub.main <= sup.main && sub.ter <= sup.ter, kErrShape, "program: incompatible levels");
    return kOk;
  };
  std::map<std::pair<int, int>, std::vector<uint32_t>> ones;  // Montgomery 1 per level
  auto mont_one = [&](const NP &np) -> const uint32_t * {
    std::vector<uint32_t> &v = ones[{np.main, np.ter}];
    if (v.empty()) {
      v.resize(np.q());
      std::vector<int> g(np.q());
      P->gidx(np, g.data());
      for (int r = 0; r < np.q(); r++) v[r] = prime::to_mont(1, P->primes[g[r]]);
    }
    return v.data();
  };

  auto rot_key_of = [&](int r, const DeviceEvk **k) -> Status {
    CHD_CHECK(rot_keys, kErrKey, "program: rotation keys missing");
    auto it = rot_keys->find(r);
    CHD_CHECK(it != rot_keys->end() && it->second, kErrKey, "program: missing rotation key " + std::to_string(r));
    *k = it->second;
    return kOk;
  };
  // MultKey (key switch + ModDown, no rescale) of register a of every
  // ciphertext into spare2
  auto mult_key_batch = [&](int a, const DeviceEvk &key) -> Status {
    const DeviceCt &a0 = R[0]->at(a);
    CHD_CHECK(!a0.has_rx && a0.np.aux == 0, kErrShape, "MultKey: ciphertext must be relinearised, no aux primes");
    const int level = P->np_to_level(a0.np);
    CHD_CHECK(level >= 0, kErrInvalidLevel, "MultKey: invalid level");
    std::vector<KSIn> ins(count);
    for (int c = 0; c < count; c++) {
      const DeviceCt &x = R[c]->at(a);
      CHD_CHECK(x.np == a0.np && !x.has_rx, kErrShape, "program: batch members at different levels");
      DeviceCt &o = R[c]->at(prog.nregs + 1);
      CHD_TRY(o.reserve(x.np, false, n));
      ins[c] = KSIn{1, x.bx, x.ax, nullptr, nullptr, o.bx, o.ax};
    }
    CHD_TRY(key_switch_fused(level, count, ins.data(), key, MDType::kModDown));
    for (int c = 0; c < count; c++) {
      DeviceCt &o = R[c]->at(prog.nregs + 1);
      o.scale = R[c]->at(a).scale;
      o.num_slots = R[c]->at(a).num_slots;
    }
    return kOk;
  };
  const bool fused_ks = n == 65536 && count > 1;

  for (const ProgOp &op : prog.ops) {
    // ---- ops that run once over the whole batch ----
    bool batched = true;
    switch (op.kind) {
      case OpKind::kRelinRescale: {
        if (!fused_ks) {
          batched = false;
          break;
        }
        CHD_CHECK(mult_key, kErrKey, "program: multiplication key missing");
        const DeviceCt &a0 = R[0]->at(op.a);
        CHD_CHECK(a0.has_rx && a0.np.aux == 0, kErrShape, "Relinearize requires a ciphertext with rx");
        const int level = P->np_to_level(a0.np);
        CHD_CHECK(level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
        const NP out_np = P->level_np(level - 1, 0);
        std::vector<KSIn> ins(count);
        for (int c = 0; c < count; c++) {
          const DeviceCt &x = R[c]->at(op.a);
          CHD_CHECK(x.np == a0.np && x.has_rx, kErrShape, "program: batch members at different levels");
          DeviceCt &t = R[c]->at(prog.nregs);
          CHD_TRY(t.reserve(out_np, false, n));
          ins[c] = KSIn{2, x.bx, x.ax, nullptr, x.rx, t.bx, t.ax};
        }
        CHD_TRY(key_switch_fused(level, count, ins.data(), *mult_key, MDType::kModDownRescale));
        for (int c = 0; c < count; c++) {
          DeviceCt &t = R[c]->at(prog.nregs);
          t.scale = R[c]->at(op.a).scale / P->rescale_prod[level];
          t.num_slots = R[c]->at(op.a).num_slots;
        }
        break;
      }
      case OpKind::kRescale:
      case OpKind::kLevelDown: {
        if (count == 1) {
          batched = false;
          break;
        }
        const DeviceCt &a0 = R[0]->at(op.a);
        CHD_CHECK(a0.np.aux == 0, kErrShape, "Rescale is not supported for ciphertexts with p primes");
        const int level = P->np_to_level(a0.np);
        CHD_CHECK(level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
        const int parts = a0.has_rx ? 3 : 2;
        std::vector<const uint32_t *> src;
        std::vector<uint32_t *> dst;
        defer = true;  // the level-down constants of all ciphertexts in few launches
        for (int c = 0; c < count; c++) {
          const DeviceCt &x = R[c]->at(op.a);
          CHD_CHECK(x.np == a0.np && x.has_rx == a0.has_rx, kErrShape, "program: batch members at different levels");
          const DeviceCt *in = &x;
          if (op.kind == OpKind::kLevelDown) {
            // times the constant 1 at this level's rescale prime product, into spare2
            DeviceCt &m = R[c]->at(prog.nregs + 1);
            CHD_TRY(check_subset(x.np, cnp.at(op.c)));
            CHD_TRY(m.reserve(x.np, x.has_rx, n));
            const uint32_t *cc = cx[op.c].data() + front_of(cnp[op.c], x.np);
            CHD_TRY(const_accum(m, x.np, parts, {{&x, 0, cc}}));
            m.scale = x.scale * prog.consts[op.c].scale;
            m.num_slots = x.num_slots;
            in = &m;
          }
          DeviceCt &t = R[c]->at(prog.nregs);
          CHD_TRY(t.reserve(P->level_np(level - 1, 0), x.has_rx, n));
          for (int p = 0; p < parts; p++) {
            src.push_back(part_of(*in, p));
            dst.push_back(part_of(t, p));
          }
          t.scale = in->scale / P->rescale_prod[level];
          t.num_slots = in->num_slots;
        }
        defer = false;
        flush_accum();
        CHD_TRY(moddown(level, MDType::kRescale, src.data(), dst.data(), static_cast<int>(src.size())));
        break;
      }
      case OpKind::kHConj: {
        if (!fused_ks) {
          batched = false;
          break;
        }
        CHD_CHECK(conj_key, kErrKey, "program: conjugation key missing");
        CHD_TRY(mult_key_batch(op.a, *conj_key));
        Alternation alternation(*this, split_streams && aux_stream != nullptr);
        for (int c = 0; c < count; c++) {
          alternation.select(c);
          CHD_TRY(permute(R[c]->at(prog.nregs), R[c]->at(prog.nregs + 1), -1));
        }
        break;
      }
      case OpKind::kHRotAdd: {
        const DeviceCt &a0 = R[0]->at(op.a);
        const int slots = a0.num_slots > 0 ? a0.num_slots : n / 2;
        int dist = op.rot % slots;
        if (dist < 0) dist += slots;
        if (!fused_ks || dist == 0) {
          batched = false;
          break;
        }
        const DeviceEvk *k = nullptr;
        CHD_TRY(rot_key_of(op.rot, &k));
        CHD_TRY(mult_key_batch(op.a, *k));
        Alternation alternation(*this, split_streams && aux_stream != nullptr);
        for (int c = 0; c < count; c++) {
          alternation.select(c);
          // res = Permute(MultKey(a)) + b (Context.cpp:800-830)
          DeviceCt &t = R[c]->at(prog.nregs);
          CHD_TRY(permute(t, R[c]->at(prog.nregs + 1), dist));
          CHD_TRY(add(t, t, R[c]->at(op.b)));
        }
        break;
      }
      case OpKind::kLinTrans: {
        if (count == 1) {
          batched = false;
          break;
        }
        CHD_CHECK(lts && op.rot >= 0 && op.rot < static_cast<int>(lts->size()) && rot_keys, kErrInvalidArg,
                  "program: linear transform missing");
        std::vector<DeviceCt *> out(count);
        std::vector<const DeviceCt *> in(count);
        for (int c = 0; c < count; c++) {
          out[c] = &R[c]->at(prog.nregs);
          in[c] = &R[c]->at(op.a);
        }
        if (keys.min_ks)
          CHD_TRY(lt_evaluate_min_ks_batch(count, out.data(), in.data(), *(*lts)[op.rot], *rot_keys));
        else
          CHD_TRY(lt_evaluate_batch(count, out.data(), in.data(), *(*lts)[op.rot], *rot_keys));
        break;
      }
      default:
        batched = false;
        break;
    }
    if (batched) {
      for (int c = 0; c < count; c++) swap_regs(R[c]->at(op.dst), R[c]->at(prog.nregs));
      continue;
    }
    // ---- ops that run per ciphertext (constant accumulations of the
    // batch joined into few launches; the element-wise ops of consecutive
    // ciphertexts, which take no scratch, alternate between the context
    // stream and its second stream so that their short launches overlap) ----
    defer = count > 1 && (op.kind == OpKind::kConstMult || op.kind == OpKind::kConstAccum);
    const bool alt = count > 1 && split_streams && aux_stream != nullptr &&
                     (op.kind == OpKind::kTensor || op.kind == OpKind::kAdd || op.kind == OpKind::kSub ||
                      op.kind == OpKind::kAddConst || op.kind == OpKind::kCopy || op.kind == OpKind::kMultImag);
    Alternation alternation(*this, alt);
    for (int bc = 0; bc < count; bc++) {
    alternation.select(bc);
    std::vector<DeviceCt> &regs = *R[bc];
    DeviceCt &spare = regs[prog.nregs], &spare2 = regs[prog.nregs + 1];
    DeviceCt &t = spare;
    bool meta = false;
    switch (op.kind) {
      case OpKind::kConstMult:
      case OpKind::kLevelDown: {
        const DeviceCt &a = regs.at(op.a);
        const int level = op.kind == OpKind::kLevelDown ? P->np_to_level(NP{a.np.main, a.np.ter, 0}) : op.level;
        const NP np = P->level_np(level);
        CHD_TRY(check_subset(np, a.np));
        CHD_TRY(check_subset(np, cnp.at(op.c)));
        DeviceCt &m = op.kind == OpKind::kLevelDown ? spare2 : t;
        CHD_TRY(m.reserve(np, a.has_rx, n));
        const uint32_t *c = cx[op.c].data() + front_of(cnp[op.c], np);
        CHD_TRY(const_accum(m, np, a.has_rx ? 3 : 2, {{&a, front_of(a.np, np), c}}));
        m.scale = a.scale * prog.consts[op.c].scale;
        m.num_slots = a.num_slots;
        if (op.kind == OpKind::kLevelDown) {
          CHD_TRY(rescale(t, m));
        }
        break;
      }
      case OpKind::kTensor: {
        const DeviceCt &a = regs.at(op.a), &b = regs.at(op.b);
        CHD_CHECK(!a.has_rx && !b.has_rx, kErrShape, "Relinearization required before MultUnsafe Ct x Ct");
        const NP np = P->level_np(op.level);
        CHD_TRY(check_subset(np, a.np));
        CHD_TRY(check_subset(np, b.np));
        CHD_TRY(t.reserve(np, true, n));
        const int fa = front_of(a.np, np), fb = front_of(b.np, np), nq = np.q();
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
          row.d0 = t.bx + static_cast<size_t>(r) * n;
          row.d1 = t.ax + static_cast<size_t>(r) * n;
          row.d2 = t.rx + static_cast<size_t>(r) * n;
          row.q = P->primes[g[r]];
          row.qinv = P->qinv[g[r]];
        }
        launch_tensor(tb, P->log_n, stream);
        t.scale = a.scale * b.scale;
        t.num_slots = std::max(a.num_slots, b.num_slots);
        break;
      }
      case OpKind::kConstAccum: {
        const NP np = P->level_np(op.level);
        std::vector<Term> terms;
        double scale = 0;
        int slots = 0;
        for (size_t i = 0; i < op.srcs.size(); i++) {
          const DeviceCt &s = regs.at(op.srcs[i]);
          CHD_TRY(check_subset(np, s.np));
          CHD_TRY(check_subset(np, cnp.at(op.cs[i])));
          terms.push_back({&s, front_of(s.np, np), cx[op.cs[i]].data() + front_of(cnp[op.cs[i]], np)});
          if (scale == 0) scale = s.scale * prog.consts[op.cs[i]].scale;
          slots = std::max(slots, s.num_slots);
        }
        bool rx = false;
        if (op.plain >= 0) {
          const DeviceCt &pl = regs.at(op.plain);
          CHD_CHECK(pl.np == np, kErrShape, "program: accumulator level mismatch");
          terms.push_back({&pl, 0, mont_one(np)});
          rx = pl.has_rx;
          if (scale == 0) scale = pl.scale;
          slots = std::max(slots, pl.num_slots);
        }
        CHD_TRY(t.reserve(np, rx, n));
        CHD_TRY(const_accum(t, np, rx ? 3 : 2, terms));
        t.scale = scale;
        t.num_slots = slots;
        break;
      }
      case OpKind::kAddConst: {
        const DeviceCt &a = regs.at(op.a);
        const NP np{a.np.main, a.np.ter, 0};
        CHD_CHECK(a.np.aux == 0, kErrShape, "program: AddConst on aux primes");
        CHD_TRY(check_subset(np, cnp.at(op.c)));
        CHD_TRY(t.reserve(np, a.has_rx, n));
        const uint32_t *c = cx[op.c].data() + front_of(cnp[op.c], np);
        // b part: a.b + c; a / r parts copied
        const int nq = np.q();
        std::vector<int> g(nq);
        P->gidx(np, g.data());
        ElemBatch eb{};
        for (int r = 0; r < nq; r++) {
          if (eb.count == kMaxElemRows) {
            launch_elementwise(ElemOp::kAddConst, eb, P->log_n, stream);
            eb.count = 0;
          }
          ElemRow &e = eb.rows[eb.count++];
          e.a = a.bx + static_cast<size_t>(r) * n;
          e.dst = t.bx + static_cast<size_t>(r) * n;
          e.q = P->primes[g[r]];
          e.qinv = P->qinv[g[r]];
          e.k = c[r];
        }
        launch_elementwise(ElemOp::kAddConst, eb, P->log_n, stream);
        const size_t bytes = static_cast<size_t>(nq) * n * 4;
        cudaMemcpyAsync(t.ax, a.ax, bytes, cudaMemcpyDeviceToDevice, stream);
        if (a.has_rx) cudaMemcpyAsync(t.rx, a.rx, bytes, cudaMemcpyDeviceToDevice, stream);
        t.scale = a.scale;
        t.num_slots = a.num_slots;
        break;
      }
      case OpKind::kAdd:
        CHD_TRY(add(t, regs.at(op.a), regs.at(op.b)));
        break;
      case OpKind::kSub:
        CHD_TRY(sub(t, regs.at(op.a), regs.at(op.b)));
        break;
      case OpKind::kRelinRescale:
        CHD_CHECK(mult_key, kErrKey, "program: multiplication key missing");
        CHD_TRY(relinearize(t, regs.at(op.a), *mult_key, true));
        break;
      case OpKind::kRescale:
        CHD_TRY(rescale(t, regs.at(op.a)));
        break;
      case OpKind::kCopy: {
        const DeviceCt &a = regs.at(op.a);
        CHD_TRY(t.reserve(a.np, a.has_rx, n));
        const size_t bytes = static_cast<size_t>(a.np.total()) * n * 4;
        for (int p = 0; p < (a.has_rx ? 3 : 2); p++)
          cudaMemcpyAsync(part_of(t, p), part_of(a, p), bytes, cudaMemcpyDeviceToDevice, stream);
        t.scale = a.scale;
        t.num_slots = a.num_slots;
        break;
      }
      case OpKind::kSetScale:
        regs.at(op.dst).scale = op.scale;
        meta = true;
        break;
      case OpKind::kSetSlots:
        regs.at(op.dst).num_slots = op.rot;
        meta = true;
        break;
      case OpKind::kHConj:
        CHD_CHECK(conj_key, kErrKey, "program: conjugation key missing");
        CHD_TRY(hconj(t, regs.at(op.a), *conj_key));
        break;
      case OpKind::kMultImag:
        CHD_TRY(mult_imag_unit(t, regs.at(op.a)));
        break;
      case OpKind::kModUpToMax:
        if (uses_sse()) {
          CHD_CHECK(keys.dts && keys.std_key, kErrKey,
                    "program: dense-to-sparse and sparse-to-dense keys required (sparse-secret encapsulation)");
          CHD_TRY(modup_to_max_sse(t, regs.at(op.a), *keys.dts, *keys.std_key));
        } else {
          CHD_TRY(modup_to_max(t, regs.at(op.a)));
        }
        break;
      case OpKind::kHRotAdd: {
        CHD_CHECK(rot_keys, kErrKey, "program: rotation keys missing");
        auto it = rot_keys->find(op.rot);
        CHD_CHECK(it != rot_keys->end() && it->second, kErrKey,
                  "program: missing rotation key " + std::to_string(op.rot));
        CHD_TRY(hrot_add(t, regs.at(op.a), regs.at(op.b), *it->second, op.rot));
        break;
      }
      case OpKind::kLinTrans:
        CHD_CHECK(lts && op.rot >= 0 && op.rot < static_cast<int>(lts->size()) && rot_keys, kErrInvalidArg,
                  "program: linear transform missing");
        if (keys.min_ks) {
          CHD_TRY(lt_evaluate_min_ks(t, regs.at(op.a), *(*lts)[op.rot], *rot_keys));
        } else {
          CHD_TRY(lt_evaluate(t, regs.at(op.a), *(*lts)[op.rot], *rot_keys));
        }
        break;
    }
    if (!meta) swap_regs(regs.at(op.dst), t);
    }
    alternation.finish();
    defer = false;
    flush_accum();
  }
  return check_cuda("program");
}

}  // namespace chd
