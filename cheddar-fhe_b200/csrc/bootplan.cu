// Bootstrapping plan: constants, CoeffToSlot / SlotToCoeff linear
// transforms and the Boot op program.
//
// Follows the reference:
//   BootContext ctor (src/extension/BootContext.cpp:38-92): scale-up
//     exponent, CtS / StC constants, EvalMod;
//   EvalSpecialFFT::PopulatePlainMatrices / PreparePlaintexts / BSGSSplit
//     (src/extension/EvalSpecialFFT.cpp:30-300): the special FFT as
//     striped butterfly stages, grouped into num_cts (num_stc) phases, each
//     a LinearTransform at its level with the min-KS pre-rotations;
//   BootContext::Boot (BootContext.cpp:296-370): scale-up at level -1,
//     ModUpToMax, CoeffToSlot, real / imaginary split, EvalMod on each,
//     recombination, SlotToCoeff.
// Any power-of-two slot count from 256 to N/2.  With fewer than N/2 slots
// (BootContext.cpp:321-360, EvalSpecialFFT.cpp:212-226, 268-282, 350-362):
// a Trace after ModUpToMax, the last CtS and the first StC phase extended
// to 2n x 2n matrices (the real and imaginary parts side by side), one
// EvalMod on HConj(x) + x, and a final HRotAdd by n.
#include <algorithm>
#include <cmath>

#include "host.h"

namespace chd {
namespace {

using cd = std::complex<double>;

int log2_ceil(int a) {
  int r = 0;
  while ((1 << r) < a) r++;
  return r;
}
bool is_pow2(int a) { return a > 0 && (a & (a - 1)) == 0; }

std::pair<int, int> bsgs_split(int num_diag) {
  // EvalSpecialFFT::BSGSSplit, EvalSpecialFFT.cpp:33-62
  if (num_diag <= 4) return {num_diag, 1};
  int bs;
  switch (num_diag) {
    case 7:
    case 8:
    case 15:
    case 16:
      bs = 4;
      break;
    case 31:
    case 32:
    case 63:
    case 64:
      bs = 8;
      break;
    default:
      bs = 1 << ((log2_ceil(num_diag) + 1) / 2);
      break;
  }
  return {bs, (num_diag + bs - 1) / bs};
}

// The 2n x 2n matrix [[D, 0], [0, D f]] in diagonal form (rotation index i
// >= n/2 moves to i + n): the last CtS phase (f = -i) and the first StC
// phase (f = i) of a sparse-slot bootstrap, EvalSpecialFFT.cpp:212-226,
// 268-282
SMat extend_sparse(const SMat &ph, int ns, cd f) {
  SMat e;
  e.h = e.w = 2 * ns;
  for (const auto &d : ph.d) {
    const int dst = d.first >= ns / 2 ? d.first + ns : d.first;
    std::vector<cd> &v = e.d.emplace(dst, std::vector<cd>(2 * ns, cd(0))).first->second;
    for (int j = 0; j < ns; j++) {
      v[j] = d.second[j];
      v[j + ns] = d.second[j] * f;
    }
  }
  return e;
}

}  // namespace

Status Context::boot_build(int num_slots, int variant, int num_cts, int num_stc, int log_msg_ratio, BootPlan *out) {
  const int half = P->n / 2;
  CHD_CHECK(num_slots >= 256 && is_pow2(num_slots), kErrInvalidArg, "Number of slots must be a power of 2, >= 256");
  CHD_CHECK(num_slots <= half, kErrInvalidArg, "num_slots exceeds max_num_slots");
  CHD_CHECK(variant >= 0 && variant <= 2, kErrInvalidArg,
            "Boot: variant must be kNormal (0), kImaginaryRemoving (1) or kMergeTwoReal (2)");
  const bool full = num_slots == half;
  CHD_CHECK(num_cts >= 2 && num_stc >= 2, kErrInvalidArg, "Boot: use at least 2 levels for CtS and StC");
  BootPlan &bp = *out;
  bp = BootPlan{};
  bp.num_slots = num_slots;
  bp.variant = variant;
  // BootParameter levels, BootParameter.cpp:25-41
  const auto &mod_co = boot_mod_coefficients();
  const int num_da = 3, initial_K = 2;
  const int em_levels = log2_ceil(static_cast<int>(mod_co.size())) + num_da;
  bp.max_level = P->max_level;
  bp.cts_start = bp.max_level;
  bp.em_start = bp.max_level - num_cts;
  bp.stc_start = bp.em_start - em_levels;
  bp.end_level = bp.stc_start - num_stc;
  CHD_CHECK(bp.end_level >= 0, kErrInvalidLevel, "Boot: not enough levels");
  CHD_CHECK(P->spec.default_encryption_level == bp.stc_start, kErrInvalidArg,
            "Parameter mismatch for BootContext (default encryption level must be the StC start level)");
  // BootContext ctor, BootContext.cpp:44-92
  auto log2_scale = [](double s) { return static_cast<int>(std::log2(s) + 0.5); };
  double level_zero_scale = P->spec.base_scale;
  const int log_lzs = log2_scale(level_zero_scale);
  const NP b = P->level_np(-1);
  std::vector<int> gb(b.q());
  P->gidx(b, gb.data());
  double q0_prod = 1.0;
  for (int g : gb) q0_prod *= P->primes[g];
  const int log_q0 = log2_scale(q0_prod);
  bp.log_scaleup = (log_q0 - log_lzs) - log_msg_ratio;
  CHD_CHECK(bp.log_scaleup >= 0, kErrInvalidArg, "Invalid level zero scaleup");
  level_zero_scale *= (1 << bp.log_scaleup);
  CHD_CHECK(log_q0 <= 62 && log_lzs <= 62, kErrInvalidArg, "Invalid q0_prod or level zero scale");
  const int log_em_start = log2_scale(P->rescale_prod.at(bp.em_start));
  const int actual_K = (1 << num_da) * initial_K;
  double em_end = static_cast<double>(uint64_t{1} << log_em_start);
  for (int i = 0; i < em_levels; i++) em_end = em_end * em_end / P->rescale_prod.at(bp.em_start - i);
  bp.cts_const = static_cast<double>(uint64_t{1} << (log_em_start - P->log_n)) / (q0_prod * actual_K);
  bp.stc_const = (q0_prod * P->scale.at(bp.end_level)) / (em_end * level_zero_scale);
  // GetStCConst(variant), BootContext.cpp:116-121
  if (variant != 0) bp.stc_const /= 2;

  // ---- special FFT stages (EvalSpecialFFT::PopulatePlainMatrices) ----
  const int ns = num_slots, M = 2 * P->n, stages = log2_ceil(ns);
  const auto &tw = enc_twiddles();
  std::vector<SMat> fft(stages), ifft(stages);
  for (int i = 0; i < stages; i++) {
    const int stride = 1 << i, sg = stride * 2, st8 = stride << 3, gap = M / st8;
    SMat &ft = fft[i];
    SMat &it = ifft[stages - i - 1];
    ft.h = ft.w = it.h = it.w = ns;
    ft.d.emplace(0, std::vector<cd>(ns, cd(0)));
    ft.d.emplace(stride, std::vector<cd>(ns, cd(0)));
    if (i != stages - 1) ft.d.emplace(ns - stride, std::vector<cd>(ns, cd(0)));
    it.d.emplace(0, std::vector<cd>(ns, cd(0)));
    it.d.emplace(stride, std::vector<cd>(ns, cd(0)));
    if (i != stages - 1) it.d.emplace(ns - stride, std::vector<cd>(ns, cd(0)));
    // at the last stage ns - stride == stride: the "minus" diagonal is the
    // "plus" one, as in the reference's map
    std::vector<cd> &f0 = ft.d[0], &fp = ft.d[stride], &fm = ft.d[ns - stride];
    std::vector<cd> &i0 = it.d[0], &ip = it.d[stride], &im = it.d[ns - stride];
    for (int j = 0; j < stride; j++) {
      const int fti = static_cast<int>(P->galois[j] % st8) * gap;
      const int iti = (st8 - static_cast<int>(P->galois[j] % st8)) * gap;
      const cd ftw = tw[fti], itw = tw[iti];
      f0[j] = 1;
      fp[j] = ftw;
      fm[j + stride] = 1;
      f0[j + stride] = -ftw;
      i0[j] = 1;
      ip[j] = 1;
      im[j + stride] = itw;
      i0[j + stride] = -itw;
    }
    const int num_double = log2_ceil(ns / sg);
    for (int r = 0; r < num_double; r++) {
      const int len = sg * (1 << r);
      auto dup = [&](std::vector<cd> &v) { std::copy(v.begin(), v.begin() + len, v.begin() + len); };
      dup(f0);
      dup(fp);
      if (i != stages - 1) dup(fm);
      dup(i0);
      dup(ip);
      if (i != stages - 1) dup(im);
    }
  }

  // ---- phases (EvalSpecialFFT::PreparePlaintexts) ----
  const double cts_div = std::pow(bp.cts_const, 1.0 / num_cts);
  const double stc_div = std::pow(bp.stc_const, 1.0 / num_stc);
  bp.lts.resize(num_cts + num_stc);
  int left = stages, cumul = 0;
  for (int i = 0; i < num_cts; i++) {
    const int st = i == 0 ? (left + num_cts - 1) / num_cts : left / (num_cts - i);
    left -= st;
    SMat ph = ifft[cumul];
    for (int j = cumul + 1; j < cumul + st; j++) ph = smat_mult(ifft[j], ph);
    if (i == num_cts - 1 && !full) ph = extend_sparse(ph, ns, cd(0, -1));
    ph = smat_scale(ph, cd(cts_div));
    int eff = static_cast<int>(ph.d.size());
    if (i == num_cts - 1) eff += 1;
    auto [bs, gs] = bsgs_split(eff);
    int pre, add = -(1 << left);
    if (i == 0) {
      pre = 1 << left;
    } else if (i == num_cts - 1) {
      pre = -(1 << st);
      add = 0;
    } else {
      pre = -((1 << st) - 1) * (1 << left);
    }
    const int lvl = bp.cts_start - i;
    CHD_TRY(lt_build(ph, lvl, P->rescale_prod.at(lvl), bs, gs, pre, add, false, &bp.lts[i]));
    cumul += st;
  }
  left = stages;
  cumul = 0;
  for (int i = 0; i < num_stc; i++) {
    const int st = left / (num_stc - i);
    left -= st;
    SMat ph = fft[cumul];
    for (int j = cumul + 1; j < cumul + st; j++) ph = smat_mult(fft[j], ph);
    if (i == 0 && !full) ph = extend_sparse(ph, ns, cd(0, 1));
    ph = smat_scale(ph, cd(stc_div));
    int eff = static_cast<int>(ph.d.size());
    if (i == 0) eff += 1;
    auto [bs, gs] = bsgs_split(eff);
    int pre, add;
    if (i == 0) {
      pre = -(1 << st);
      add = 1 << st;
    } else if (i == num_stc - 1) {
      pre = 1 << cumul;
      add = 0;
    } else {
      pre = -((1 << st) - 1) * (1 << cumul);
      add = 1 << (st + cumul);
    }
    const int lvl = bp.stc_start - i;
    CHD_TRY(lt_build(ph, lvl, P->rescale_prod.at(lvl), bs, gs, pre, add, false, &bp.lts[num_cts + i]));
    cumul += st;
  }
  for (auto &l : bp.lts) bp.lt_ptrs.push_back(&l);
  {
    std::vector<int> r;
    for (const auto &l : bp.lts) {
      for (int x : l.bs_idx)
        if (x) r.push_back(x);
      for (int x : l.gs_idx)
        if (x) r.push_back(x);
    }
    // AddRequiredRotations, BootContext.cpp:175-184 and
    // EvalSpecialFFT.cpp:323-325: Trace distances n, 2n, .., N/4 and the
    // StC fold by n
    if (!full)
      for (int d = ns; d < half; d *= 2) bp.extra_rotations.push_back(d);
    for (int x : bp.extra_rotations) r.push_back(x);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    bp.rotations = r;
  }

  // ---- the Boot program (BootContext::Boot, full slots, kNormal) ----
  Program &pg = bp.prog;
  pg.input = pg.reg();
  auto op = [&](OpKind k, int a, int b = -1) {
    ProgOp o;
    o.kind = k;
    o.dst = pg.reg();
    o.a = a;
    o.b = b;
    pg.ops.push_back(o);
    return o.dst;
  };
  // 0. scale up: MultUnsafe(input, scaleup constant, level -1)
  const int su = pg.add_const(-1, 1.0, static_cast<double>(1 << bp.log_scaleup));
  {
    ProgOp o;
    o.kind = OpKind::kConstMult;
    o.dst = pg.reg();
    o.a = pg.input;
    o.c = su;
    o.level = -1;
    pg.ops.push_back(o);
    // 1. ModUpToMax (with sparse-secret encapsulation when the parameters
    // have it), then the Trace over the N/2 slots (BootContext::Trace,
    // BootContext.cpp:368-400): x += HRot(x, n 2^i) for i < log2(N / 2n)
    int x = op(OpKind::kModUpToMax, o.dst);
    auto set_slots = [&](int reg, int slots) {
      ProgOp m;
      m.kind = OpKind::kSetSlots;
      m.dst = reg;
      m.a = reg;
      m.rot = slots;
      pg.ops.push_back(m);
    };
    auto hrot_add = [&](int a, int rot) {
      ProgOp h;
      h.kind = OpKind::kHRotAdd;
      h.dst = pg.reg();
      h.a = a;
      h.b = a;
      h.rot = rot;
      pg.ops.push_back(h);
      return h.dst;
    };
    if (!full) {
      set_slots(x, half);
      for (int d = ns; d < half; d *= 2) x = hrot_add(x, d % half);
      set_slots(x, ns);
    }
    // 2. CoeffToSlot
    for (int i = 0; i < num_cts; i++) {
      ProgOp l;
      l.kind = OpKind::kLinTrans;
      l.dst = pg.reg();
      l.a = x;
      l.rot = i;
      pg.ops.push_back(l);
      x = l.dst;
    }
    if (!full) set_slots(x, 2 * ns);
    // 3. real / imaginary parts, EvalMod on each (full slots), or both
    // parts side by side in 2n slots: EvalMod(HConj(x) + x)
    int em_reg = -1, em_level = 0;
    double s0 = 0, s1 = 0;
    {
      // the EvalMod start scale is fixed by the parameters; set it first
      Program probe;
      probe.input = probe.reg();
      CHD_TRY(compile_evalmod(probe, probe.input, bp.em_start, mod_co, num_da, initial_K, &em_reg, &em_level, &s0,
                              &s1));
    }
    bp.em_start_scale = s0;
    bp.em_end_scale = s1;
    ProgOp ss;
    ss.kind = OpKind::kSetScale;
    ss.dst = x;
    ss.a = x;
    ss.scale = s0;
    pg.ops.push_back(ss);
    const int conj = op(OpKind::kHConj, x);
    if (full) {
      int re = op(OpKind::kAdd, x, conj);
      int im = op(OpKind::kSub, conj, x);
      im = op(OpKind::kMultImag, im);
      int re_out = -1, im_out = -1;
      CHD_TRY(compile_evalmod(pg, re, bp.em_start, mod_co, num_da, initial_K, &re_out, &em_level, &s0, &s1));
      CHD_TRY(compile_evalmod(pg, im, bp.em_start, mod_co, num_da, initial_K, &im_out, &em_level, &s0, &s1));
      im_out = op(OpKind::kMultImag, im_out);
      x = op(OpKind::kAdd, re_out, im_out);
    } else {
      // HConjAdd(res, x, x) = HConj(x) + x (Context.cpp:836-860)
      const int merged = op(OpKind::kAdd, conj, x);
      CHD_TRY(compile_evalmod(pg, merged, bp.em_start, mod_co, num_da, initial_K, &x, &em_level, &s0, &s1));
    }
    CHD_CHECK(em_level == bp.stc_start, kErrInvalidLevel, "Boot: EvalMod level bookkeeping mismatch");
    // 4. SlotToCoeff
    for (int i = 0; i < num_stc; i++) {
      ProgOp l;
      l.kind = OpKind::kLinTrans;
      l.dst = pg.reg();
      l.a = x;
      l.rot = num_cts + i;
      pg.ops.push_back(l);
      x = l.dst;
    }
    if (!full) {
      // EvaluateStC, EvalSpecialFFT.cpp:350-362: fold the two halves
      set_slots(x, 2 * ns);
      x = hrot_add(x, ns);
      set_slots(x, ns);
    }
    if (variant == 1) {
      // kImaginaryRemoving: res = HConj(res) + res (BootContext.cpp:354-357)
      const int c = op(OpKind::kHConj, x);
      x = op(OpKind::kAdd, c, x);
    }
    bp.final_scale = P->scale.at(bp.end_level);
    ProgOp fs;
    fs.kind = OpKind::kSetScale;
    fs.dst = x;
    fs.a = x;
    fs.scale = bp.final_scale;
    pg.ops.push_back(fs);
    pg.output = x;
  }
  return kOk;
}

Status Context::boot_run(const BootPlan &bp, DeviceCt &res, const DeviceCt &in, const ProgKeys &keys,
                         std::vector<DeviceCt> *regs_io) {
  std::vector<DeviceCt> local;
  std::vector<DeviceCt> *regs = regs_io ? regs_io : &local;
  DeviceCt *r = &res;
  const DeviceCt *i = &in;
  return boot_run_batch(bp, 1, &r, &i, keys, &regs);
}

Status Context::boot_run_batch(const BootPlan &bp, int count, DeviceCt *const *res, const DeviceCt *const *in,
                               const ProgKeys &keys, std::vector<DeviceCt> *const *regs) {
  // BootContext::Boot (BootContext.cpp:296-370) on `count` ciphertexts with
  // the program's key switches, rescales and linear transforms batched
  // across them; an input above level 0 is first brought down with
  // Context::LevelDown (Context.cpp:917-929): per level, times the constant 1
  // at that level's scale, then Rescale
  CHD_CHECK(count >= 1, kErrInvalidArg, "Boot: empty batch");
  CHD_CHECK(keys.mult && keys.conj && keys.rot, kErrKey, "Boot: multiplication, conjugation and rotation keys needed");
  for (int c = 0; c < count; c++) {
    CHD_CHECK(in[c]->np.aux == 0 && !in[c]->has_rx, kErrShape, "Boot: input must be relinearised without aux primes");
    const int in_level = P->np_to_level(in[c]->np);
    CHD_CHECK(in_level >= 0 && in_level <= P->spec.default_encryption_level, kErrInvalidLevel,
              "Boot: input level must be in [0, default encryption level]");
    // GetBootEnabledNumSlots (BootContext.cpp:124-147): the input's slots
    // must fit the prepared slot count (a smaller power of two is periodic
    // in it)
    const int in_slots = in[c]->num_slots > 0 ? in[c]->num_slots : P->n / 2;
    CHD_CHECK(in_slots <= bp.num_slots, kErrInvalidArg,
              "Boot: not prepared for " + std::to_string(in_slots) + " slots (prepared: " +
                  std::to_string(bp.num_slots) + ")");
    for (int d = 0; d < c; d++) CHD_CHECK(regs[c] != regs[d], kErrInvalidArg, "Boot: batch members share registers");
  }
  for (int c = 0; c < count; c++) {
    std::vector<DeviceCt> &rg = *regs[c];
    CHD_TRY(program_regs(bp.prog, rg));
    DeviceCt &r0 = rg[bp.prog.input];
    const DeviceCt &x = *in[c];
    const int in_level = P->np_to_level(x.np);
    CHD_TRY(r0.reserve(x.np, false, P->n));
    const size_t bytes = static_cast<size_t>(x.np.total()) * P->n * 4;
    cudaMemcpyAsync(r0.bx, x.bx, bytes, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(r0.ax, x.ax, bytes, cudaMemcpyDeviceToDevice, stream);
    r0.scale = x.scale;
    r0.num_slots = x.num_slots;
    if (in_level > 0) {
      Program ld;
      ld.input = ld.reg();
      int y = ld.input;
      for (int i = in_level; i > 0; i--) {
        ProgOp m;
        m.kind = OpKind::kConstMult;
        m.dst = ld.reg();
        m.a = y;
        m.c = ld.add_const(i, P->scale.at(i), 1.0);
        m.level = i;
        ld.ops.push_back(m);
        ProgOp r;
        r.kind = OpKind::kRescale;
        r.dst = ld.reg();
        r.a = m.dst;
        ld.ops.push_back(r);
        y = r.dst;
      }
      ld.output = y;
      std::vector<DeviceCt> lregs;
      CHD_TRY(program_regs(ld, lregs));
      swap_regs(lregs[ld.input], r0);
      CHD_TRY(run_program(ld, lregs, keys, nullptr));
      swap_regs(lregs[ld.output], r0);
    }
  }
  CHD_TRY(run_program_batch(bp.prog, count, regs, keys, &bp.lt_ptrs));
  for (int c = 0; c < count; c++) {
    const DeviceCt &o = (*regs[c])[bp.prog.output];
    const int in_slots = in[c]->num_slots;
    CHD_TRY(res[c]->reserve(o.np, false, P->n));
    const size_t ob = static_cast<size_t>(o.np.total()) * P->n * 4;
    cudaMemcpyAsync(res[c]->bx, o.bx, ob, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(res[c]->ax, o.ax, ob, cudaMemcpyDeviceToDevice, stream);
    res[c]->scale = bp.final_scale;
    res[c]->num_slots = in_slots;
  }
  return check_cuda("boot");
}

}  // namespace chd
