// Polynomial evaluation and EvalMod, compiled to an op program.
//
// The planning follows src/extension/EvalPoly.cpp and EvalMod.cpp of the
// reference step by step, so the constants (values, levels and FP64 scales)
// and the operations are the reference's:
//   * EvalPoly: coefficient clean-up (RemoveZero), odd/even/normal type,
//     the recursive split tree (EvalPolyNode: power-of-two split, Chebyshev
//     fold-back low[s - i] -= high[i], high[i] *= 2, leaves below the
//     baby-step threshold), the basis T_k built by BasisMap::AddBase with
//     AXYPBZ nodes (T_(l+r) = 2 T_l T_r - T_(l-r)), lazy rescaling of the
//     low halves;
//   * EvalMod: x - 1/(4K) then the Chebyshev cosine polynomial, then the
//     double-angle steps 2 x^2 - c.
// Evaluation emits: kConstMult / kTensor (MultUnsafe), kConstAccum (CAccum,
// leaf sums and the AXYPBZ z term), kAddConst, kAdd, kRelinRescale,
// kRescale, kLevelDown (MultiLevelCiphertext::AddLowerLevelsUntil).
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <set>

#include "host.h"

namespace chd {
namespace {

constexpr double kZeroCoeff = 1e-9;  // kZeroCoeffThreshold, EvalPoly.h

int log2_ceil(int a) {
  int r = 0;
  while ((1 << r) < a) r++;
  return r;
}
int log2_floor(int a) {
  int r = 0;
  while ((2 << r) <= a) r++;
  return r;
}
bool is_pow2(int a) { return a > 0 && (a & (a - 1)) == 0; }

void remove_zero(std::vector<double> &c) {
  // RemoveZero, EvalPoly.cpp:10-21
  while (!c.empty() && std::fabs(c.back()) < kZeroCoeff) c.pop_back();
  for (auto &x : c)
    if (std::fabs(x) < kZeroCoeff) x = 0;
}

enum class PolyType { kOdd, kEven, kNormal };

struct Compiler;

// AXYPBZ (EvalPoly.cpp:109-236): a x y + b z (with z) or a x y + b
struct Axypbz {
  int a = 1;
  double b = 0;
  bool has_a = false, has_b = false, has_z = false;
  int a_c = -1, b_c = -1;
  int x_level = 0, y_level = 0, z_level = 0;
  double x_scale = 0, y_scale = 0, z_scale = 0;
  int final_level = 0;
  double final_scale = 0;
};

// multi-level ciphertext: one register per level (MultiLevelCiphertext)
struct MLReg {
  std::map<int, int> at;  // level -> register
  int max_level() const { return at.rbegin()->first; }
  int min_level() const { return at.begin()->first; }
};

struct Compiler {
  Context &C;
  Program &prog;
  PolyType type = PolyType::kNormal;
  bool cheb = true;
  int input_level = 0;
  double input_scale = 0;
  std::map<int, Axypbz> basis;  // BasisMap::basis_eval_
  std::map<int, MLReg> regs;    // evaluated bases by degree
  std::map<int, int> level_down_c;

  double rescale_prod(int level) const { return C.P->rescale_prod.at(level); }

  int split_base(int d) const {
    // BasisMap::SplitBaseDegree, EvalPoly.cpp:248-260
    int split;
    if (is_pow2(d))
      split = d / 2;
    else if (type == PolyType::kEven)
      split = 1 << log2_floor(d);
    else
      split = (1 << log2_floor(d)) - 1;
    return std::max(split, d - split);
  }
  bool exists(int d) const { return d == 1 || basis.count(d); }
  std::pair<int, double> base_ls(int d) const {
    if (d == 1) return {input_level, input_scale};
    const Axypbz &e = basis.at(d);
    return {e.final_level, e.final_scale};
  }

  Status make_axypbz(Axypbz &e, int a, double b, int xl, double xs, int yl, double ys, bool has_z, int zl,
                     double zs) {
    // AXYPBZ constructors, EvalPoly.cpp:125-193
    e.a = a;
    e.b = b;
    e.has_z = has_z;
    e.x_level = xl;
    e.x_scale = xs;
    e.y_level = yl;
    e.y_scale = ys;
    e.z_level = has_z ? zl : 0;
    e.z_scale = has_z ? zs : 0;
    const double working_scale = xs * ys;
    int working_level = std::min(xl, yl);
    if (has_z) working_level = std::min(working_level, zl);
    CHD_CHECK(working_level >= 1, kErrInvalidLevel, "AXYPBZ: Invalid levels");
    CHD_CHECK(C.mult_unsafe_compatible(xl, working_level) && C.mult_unsafe_compatible(yl, working_level),
              kErrInvalidLevel, "AXYPBZ: Invalid levels");
    if (b == 0.0) {
      e.has_b = false;
    } else {
      e.has_b = true;
      if (has_z) {
        CHD_CHECK(C.mult_unsafe_compatible(zl, working_level), kErrInvalidLevel, "AXYPBZ: Invalid levels");
        const double b_scale = working_scale / zs;
        e.b_c = prog.add_const(working_level, b_scale, b);
      } else {
        e.b_c = prog.add_const(working_level, working_scale, b);
      }
    }
    CHD_CHECK(a != 0, kErrInvalidArg, "AXYPBZ: a should not be 0");
    e.has_a = a != 1;
    if (e.has_a) e.a_c = prog.add_const(working_level, 1.0, a);
    e.final_level = working_level - 1;
    e.final_scale = working_scale / rescale_prod(working_level);
    return kOk;
  }

  Status add_base(int d) {
    // BasisMap::AddBase, EvalPoly.cpp:277-350
    CHD_CHECK(d >= 2, kErrInvalidArg, "AddBase: base degree should be at least 2");
    const int left = split_base(d), right = d - left;
    if (!exists(left)) CHD_TRY(add_base(left));
    if (!exists(right)) CHD_TRY(add_base(right));
    auto [ll, ls] = base_ls(left);
    auto [rl, rs] = base_ls(right);
    const int working = std::min(ll, rl);
    while (!C.mult_unsafe_compatible(ll, working)) ll -= 1;
    while (!C.mult_unsafe_compatible(rl, working)) rl -= 1;
    Axypbz e;
    if (cheb) {
      const int sub = left - right;
      if (sub == 0) {
        CHD_TRY(make_axypbz(e, 2, -1, ll, ls, rl, rs, false, 0, 0));
      } else {
        if (!exists(sub)) CHD_TRY(add_base(sub));
        auto [sl, ss] = base_ls(sub);
        while (!C.mult_unsafe_compatible(sl, working)) sl -= 1;
        CHD_TRY(make_axypbz(e, 2, -1, ll, ls, rl, rs, true, sl, ss));
      }
    } else {
      CHD_TRY(make_axypbz(e, 1, 0, ll, ls, rl, rs, false, 0, 0));
    }
    basis.emplace(d, e);
    return kOk;
  }

  // ---- emission helpers ----
  int level_down_const(int level) {
    auto it = level_down_c.find(level);
    if (it != level_down_c.end()) return it->second;
    // MultiLevelCiphertext::StaticInit: 1.0 at the rescale prime product
    const int c = prog.add_const(level, rescale_prod(level), 1.0);
    level_down_c[level] = c;
    return c;
  }
  Status add_lower_levels_until(MLReg &ml, int min_level) {
    // Context::AddLowerLevelsUntil, Context.cpp:931-949
    if (ml.at.count(min_level)) return kOk;
    CHD_CHECK(min_level <= ml.max_level() && min_level >= 0, kErrInvalidLevel, "AddLowerLevelsUntil: invalid level");
    for (int i = ml.min_level() - 1; i >= min_level; i--) {
      ProgOp op;
      op.kind = OpKind::kLevelDown;
      op.a = ml.at.at(i + 1);
      op.dst = prog.reg();
      op.level = i + 1;
      op.c = level_down_const(i + 1);
      prog.ops.push_back(op);
      ml.at[i] = op.dst;
    }
    return kOk;
  }
  Status base_at(int d, int working_level, int *reg, int *level) {
    MLReg &ml = regs.at(d);
    int l = ml.max_level();
    while (!C.mult_unsafe_compatible(l, working_level)) l -= 1;
    CHD_TRY(add_lower_levels_until(ml, l));
    *reg = ml.at.at(l);
    *level = l;
    return kOk;
  }

  Status eval_axypbz(const Axypbz &e, int x, int y, int z, int *out) {
    // AXYPBZ::Evaluate, EvalPoly.cpp:195-236
    const int wl = e.final_level + 1;
    int t = prog.reg();
    if (e.has_a) {
      ProgOp m;
      m.kind = OpKind::kConstMult;
      m.dst = t;
      m.a = x;
      m.c = e.a_c;
      m.level = wl;
      prog.ops.push_back(m);
      ProgOp tz;
      tz.kind = OpKind::kTensor;
      tz.dst = t;
      tz.a = t;
      tz.b = y;
      tz.level = wl;
      prog.ops.push_back(tz);
    } else {
      ProgOp tz;
      tz.kind = OpKind::kTensor;
      tz.dst = t;
      tz.a = x;
      tz.b = y;
      tz.level = wl;
      prog.ops.push_back(tz);
    }
    if (e.has_b) {
      if (e.has_z) {
        ProgOp ca;
        ca.kind = OpKind::kConstAccum;
        ca.dst = t;
        ca.srcs = {z};
        ca.cs = {e.b_c};
        ca.plain = t;
        ca.level = wl;
        prog.ops.push_back(ca);
      } else {
        ProgOp ac;
        ac.kind = OpKind::kAddConst;
        ac.dst = t;
        ac.a = t;
        ac.c = e.b_c;
        prog.ops.push_back(ac);
      }
    }
    ProgOp rr;
    rr.kind = OpKind::kRelinRescale;
    rr.dst = prog.reg();
    rr.a = t;
    prog.ops.push_back(rr);
    *out = rr.dst;
    return kOk;
  }

  Status eval_basis(int in) {
    // BasisMap::Evaluate, EvalPoly.cpp:352-383
    regs[1].at[input_level] = in;
    for (const auto &be : basis) {
      const int d = be.first;
      const Axypbz &e = be.second;
      const int left = split_base(d), right = d - left, sub = left - right;
      CHD_TRY(add_lower_levels_until(regs.at(left), e.x_level));
      CHD_TRY(add_lower_levels_until(regs.at(right), e.y_level));
      const int x = regs.at(left).at.at(e.x_level), y = regs.at(right).at.at(e.y_level);
      int out = -1;
      if (cheb && sub != 0) {
        CHD_TRY(add_lower_levels_until(regs.at(sub), e.z_level));
        CHD_TRY(eval_axypbz(e, x, y, regs.at(sub).at.at(e.z_level), &out));
      } else {
        CHD_TRY(eval_axypbz(e, x, y, -1, &out));
      }
      regs[d].at[e.final_level] = out;
    }
    return kOk;
  }
};

// EvalPolyNode, EvalPoly.cpp:404-705
struct Node {
  std::shared_ptr<Node> low, high;
  bool low_zero = false, low_const = false, high_const = false;
  int low_c = -1, high_c = -1;
  int split = 0;
  std::vector<double> co;
  std::map<int, int> leaf_c;  // base degree -> constant (-1 until compiled)
  int target_level = 0;
  bool do_rescale = true;

  Node(const std::vector<double> &c, int level_margin, int baby, bool cheb) : co(c) {
    const int degree = static_cast<int>(c.size()) - 1;
    const int leaf_levels = log2_ceil(degree) + 1;
    if (degree < baby && leaf_levels <= level_margin) {
      for (int i = 0; i <= degree; i++)
        if (std::fabs(c[i]) > kZeroCoeff) leaf_c[i] = -1;
      return;
    }
    split = 1 << log2_floor(degree);
    std::vector<double> lo(c.begin(), c.begin() + split), hi(c.begin() + split, c.end());
    if (cheb) {
      const int hs = static_cast<int>(hi.size());
      for (int i = 1; i < hs; i++) {
        lo[split - i] -= hi[i];
        hi[i] *= 2;
      }
    }
    remove_zero(lo);
    remove_zero(hi);
    low_zero = lo.empty();
    low_const = lo.size() <= 1;
    high_const = hi.size() == 1;
    if (!low_const) low = std::make_shared<Node>(lo, level_margin, baby, cheb);
    if (!high_const) high = std::make_shared<Node>(hi, level_margin - 1, baby, cheb);
  }
  bool is_leaf() const { return high == nullptr && !high_const; }
  void required(std::set<int> &s) const {
    for (const auto &e : leaf_c) s.insert(e.first);
    if (low) low->required(s);
    if (high) high->required(s);
    s.insert(split);
  }
  Status compile(Compiler &cp, int target, double target_scale, bool rescale) {
    // EvalPolyNode::Compile, EvalPoly.cpp:473-520
    target_level = target;
    do_rescale = rescale;
    int wl = target;
    double ws = target_scale;
    if (rescale) {
      wl = target + 1;
      ws = target_scale * cp.rescale_prod(wl);
    }
    if (low_const && !low_zero) {
      low_c = cp.prog.add_const(wl, ws, co[0]);
    } else if (low) {
      CHD_TRY(low->compile(cp, wl, ws, false));
    }
    if (high_const || high) {
      const double split_scale = cp.base_ls(split).second;
      const double high_scale = ws / split_scale;
      // the reference passes (scale, level) swapped to EncodeConstant here
      // (EvalPoly.cpp:503-505), which no valid parameter set survives
      CHD_CHECK(!high_const, kErrUnsupported, "EvalPoly: constant high part is not supported");
      CHD_TRY(high->compile(cp, wl, high_scale, true));
    }
    for (auto &e : leaf_c) {
      const double value = co[e.first];
      double scale = ws;
      if (e.first != 0) scale /= cp.base_ls(e.first).second;
      e.second = cp.prog.add_const(wl, scale, value);
    }
    return kOk;
  }
  Status evaluate(Compiler &cp, int *res) {
    return is_leaf() ? evaluate_leaf(cp, res, false) : evaluate_middle(cp, res);
  }
  Status evaluate_middle(Compiler &cp, int *res) {
    // EvalPolyNode::EvaluateMiddleNode, EvalPoly.cpp:534-589
    Program &pg = cp.prog;
    const int wl = target_level + (do_rescale ? 1 : 0);
    int sreg = -1, slevel = 0;
    CHD_TRY(cp.base_at(split, wl, &sreg, &slevel));
    int accum = -1;
    if (high) {
      int h = -1;
      CHD_TRY(high->evaluate(cp, &h));
      ProgOp t;
      t.kind = OpKind::kTensor;
      t.dst = pg.reg();
      t.a = h;
      t.b = sreg;
      t.level = wl;
      pg.ops.push_back(t);
      accum = t.dst;
    } else {
      ProgOp m;
      m.kind = OpKind::kConstMult;
      m.dst = pg.reg();
      m.a = sreg;
      m.c = high_c;
      m.level = wl;
      pg.ops.push_back(m);
      accum = m.dst;
    }
    if (low) {
      if (low->is_leaf()) {
        CHD_TRY(low->evaluate_leaf(cp, &accum, true));
      } else {
        int t2 = -1;
        CHD_TRY(low->evaluate(cp, &t2));
        ProgOp a;
        a.kind = OpKind::kAdd;
        a.dst = accum;
        a.a = accum;
        a.b = t2;
        pg.ops.push_back(a);
      }
    } else if (low_const && !low_zero) {
      ProgOp a;
      a.kind = OpKind::kAddConst;
      a.dst = accum;
      a.a = accum;
      a.c = low_c;
      pg.ops.push_back(a);
    }
    if (do_rescale) {
      // accum carries Rx exactly when it came from a tensor product
      ProgOp r;
      r.kind = high ? OpKind::kRelinRescale : OpKind::kRescale;
      r.dst = pg.reg();
      r.a = accum;
      pg.ops.push_back(r);
      *res = r.dst;
    } else {
      *res = accum;
    }
    return kOk;
  }
  Status evaluate_leaf(Compiler &cp, int *res, bool inplace) {
    // EvalPolyNode::EvaluateLeaf, EvalPoly.cpp:591-672
    Program &pg = cp.prog;
    CHD_CHECK(!(do_rescale && inplace), kErrInvalidArg, "Rescale and inplace EvaluateLeaf is not compatible");
    const int wl = target_level + (do_rescale ? 1 : 0);
    ProgOp ca;
    ca.kind = OpKind::kConstAccum;
    ca.level = wl;
    int zero_c = -1;
    for (const auto &e : leaf_c) {
      if (e.first == 0) {
        zero_c = e.second;
        continue;
      }
      int r = -1, l = 0;
      CHD_TRY(cp.base_at(e.first, wl, &r, &l));
      ca.srcs.push_back(r);
      ca.cs.push_back(e.second);
    }
    if (inplace) {
      ca.dst = *res;
      ca.plain = *res;
    } else {
      ca.dst = pg.reg();
    }
    int accum = ca.dst;
    if (!ca.srcs.empty() || inplace) pg.ops.push_back(ca);
    CHD_CHECK(!ca.srcs.empty() || inplace || zero_c >= 0, kErrInvalidArg, "EvalPoly: empty leaf");
    if (zero_c >= 0) {
      ProgOp a;
      a.kind = OpKind::kAddConst;
      a.dst = accum;
      a.a = accum;
      a.c = zero_c;
      pg.ops.push_back(a);
    }
    if (do_rescale) {
      ProgOp r;
      r.kind = OpKind::kRescale;
      r.dst = pg.reg();
      r.a = accum;
      pg.ops.push_back(r);
      *res = r.dst;
    } else {
      *res = accum;
    }
    return kOk;
  }
};

}  // namespace

bool Context::mult_unsafe_compatible(int l1, int l2) const {
  // Context::IsMultUnsafeCompatible, Context.cpp:356-367
  if (l1 == l2) return true;
  const NP lo = P->level_np(std::min(l1, l2)), hi = P->level_np(std::max(l1, l2));
  return lo.main <= hi.main && lo.ter <= hi.ter;
}

Status Context::compile_poly(Program &prog, int in, const std::vector<double> &coeffs, int input_level,
                             double input_scale, double target_scale, bool chebyshev, int *out_reg, int *out_level) {
  // EvalPoly ctor + DetermineType + Compile + Evaluate, EvalPoly.cpp:707-854
  std::vector<double> co = coeffs;
  remove_zero(co);
  const int degree = static_cast<int>(co.size()) - 1;
  CHD_CHECK(degree >= 2, kErrInvalidArg, "Use EvalPoly for at least >= 2 degree poly.");
  bool odd = true, even = true;
  for (int i = 0; i <= degree; i += 2)
    if (co[i] != 0) odd = false;
  for (int i = 1; i <= degree; i += 2)
    if (co[i] != 0) even = false;
  CHD_CHECK(!(even && odd), kErrInvalidArg, "Invalid polynomial type.");
  Compiler cp{*this, prog};
  cp.type = even ? PolyType::kEven : (odd ? PolyType::kOdd : PolyType::kNormal);
  cp.cheb = chebyshev;
  cp.input_level = input_level;
  cp.input_scale = input_scale;
  const int consumption = log2_ceil(degree + 1);
  const int baby = 1 << ((consumption + 1) / 2);
  Node root(co, consumption, baby, chebyshev);
  std::set<int> req;
  root.required(req);
  for (int d : req)
    if (d != 0 && d != 1) CHD_TRY(cp.add_base(d));
  const int target_level = input_level - consumption;
  CHD_CHECK(target_level >= 0, kErrInvalidLevel, "EvalPoly: not enough levels");
  CHD_TRY(root.compile(cp, target_level, target_scale, true));
  // evaluation: the input is copied into the basis (EvalPoly::Evaluate)
  int cin = prog.reg();
  ProgOp cpy;
  cpy.kind = OpKind::kCopy;
  cpy.dst = cin;
  cpy.a = in;
  prog.ops.push_back(cpy);
  CHD_TRY(cp.eval_basis(cin));
  int res = -1;
  CHD_TRY(root.evaluate(cp, &res));
  ProgOp ss;
  ss.kind = OpKind::kSetScale;
  ss.dst = res;
  ss.a = res;
  ss.scale = target_scale;
  prog.ops.push_back(ss);
  *out_reg = res;
  *out_level = target_level;
  return kOk;
}

Status Context::compile_evalmod(Program &prog, int in, int start_level, const std::vector<double> &mod_coeffs,
                                int num_double_angle, int initial_K, int *out_reg, int *out_level,
                                double *start_scale_out, double *end_scale_out) {
  // EvalMod ctor + Evaluate, EvalMod.cpp:9-61
  const int da_ratio = 1 << num_double_angle;
  const int first_log_scale = static_cast<int>(std::log2(P->rescale_prod.at(start_level)) + 0.5);
  CHD_CHECK(first_log_scale <= 62, kErrInvalidArg, "Invalid eval_mod_scale");
  const double start_scale = static_cast<double>(uint64_t{1} << first_log_scale);
  const int actual_K = (1 << num_double_angle) * initial_K;
  const int init_c = prog.add_const(start_level, start_scale, -0.25 / actual_K);
  const int mod_levels = log2_ceil(static_cast<int>(mod_coeffs.size()));
  double target_scale = start_scale;
  for (int i = 0; i < mod_levels; i++)
    target_scale = target_scale * target_scale / P->rescale_prod.at(start_level - i);
  // res = input + initial constant
  const int x = prog.reg();
  ProgOp ac;
  ac.kind = OpKind::kAddConst;
  ac.dst = x;
  ac.a = in;
  ac.c = init_c;
  prog.ops.push_back(ac);
  int reg = -1, level = 0;
  CHD_TRY(compile_poly(prog, x, mod_coeffs, start_level, start_scale, target_scale, true, &reg, &level));
  double sqrt2pi = std::pow(0.5 / M_PI, 1.0 / da_ratio);
  for (int i = 0; i < num_double_angle; i++) {
    sqrt2pi *= sqrt2pi;
    const int da_level = start_level - mod_levels - i;
    CHD_CHECK(da_level == level, kErrInvalidLevel, "EvalMod: level bookkeeping mismatch");
    // AXYPBZ(context, 2, -sqrt2pi, l, s, l, s): 2 x x - sqrt2pi
    Compiler cp{*this, prog};
    Axypbz e;
    CHD_TRY(cp.make_axypbz(e, 2, -sqrt2pi, da_level, target_scale, da_level, target_scale, false, 0, 0));
    int out = -1;
    CHD_TRY(cp.eval_axypbz(e, reg, reg, -1, &out));
    ProgOp ss;
    ss.kind = OpKind::kSetScale;
    ss.dst = out;
    ss.a = out;
    ss.scale = e.final_scale;
    prog.ops.push_back(ss);
    reg = out;
    level = e.final_level;
    target_scale = target_scale * target_scale / P->rescale_prod.at(da_level);
  }
  *out_reg = reg;
  *out_level = level;
  if (start_scale_out) *start_scale_out = start_scale;
  if (end_scale_out) *end_scale_out = target_scale;
  return kOk;
}

}  // namespace chd
