// The 64-bit word path: the reference's Context<uint64_t> instantiation
// (src/core/NTT.cu:1313, ModSwitch.cu:688, ElementWise.cu:1706,
// Context.cpp:952) for parameter sets with primes up to 2^62, e.g. the
// reference's bootparam_40_64bit.json (40-55-bit main primes, 56-bit
// auxiliary primes).  The same algorithms as the 32-bit path with R = 2^64:
// residues in the Montgomery form x 2^64 mod q, bit-reversed evaluation
// domain, prime order terminal reversed / main / auxiliary, BConv tables
// q-hat R^2 mod p centred.  N = 2^16; the evaluation core only (NTT, ModUp,
// ModDown, Rescale, ModDownAndRescale, HMult with relinearisation and
// rescale, HRot), with unfused launches.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "host.h"

namespace chd {
namespace w64 {

using u64 = uint64_t;
using i64 = int64_t;
using u128 = unsigned __int128;
using i128 = __int128;
using MDType = Context::MDType;

// ---- prime utilities (include/common/PrimeUtils.h with word = uint64_t) ----
u64 mul_mod(u64 a, u64 b, u64 q);
u64 pow_mod(u64 a, int64_t e, u64 q);
u64 inv_mod(u64 a, u64 q);
u64 smallest_generator(u64 q);
u64 primitive_root(u64 m, u64 q);
i64 inv_mod_word(u64 q);  // q^-1 mod 2^64, signed
u64 to_mont(u64 a, u64 q);
i64 centre(u64 a, u64 q);

// ---- level model ------------------------------------------------------------
class Params64 {
 public:
  static std::unique_ptr<Params64> create(const ParamSpec64 &spec, std::string *err);
  ParamSpec64 spec;
  int log_n = 0, n = 0, L = 0, alpha = 0, max_ter = 0, max_main = 0, max_level = 0;
  NP short_np;
  std::vector<u64> primes;  // ter reversed, main, aux
  std::vector<i64> qinv;
  std::vector<double> rescale_prod;
  std::vector<double> scale;  // per level up to the default encryption level
  NP level_np(int level, int num_aux = 0) const;
  int np_to_level(const NP &np) const;
  void gidx(const NP &np, int *out) const;
  u64 galois_of(int amount) const;  // amount in [0, N/2] or -1
};

// Per-level ModSwitch constants (ModSwitch.cu:175-411 with word = uint64_t)
struct LevelMS64 {
  int level = 0, num_aux = 0, beta = 0, num_q = 0;
  std::vector<u64> mod_up1;
  std::vector<int> dig_s, dig_e;
  std::vector<std::vector<i64>> mod_up2;
  std::vector<u64> mod_down1, inv_p_prod;
  std::vector<i64> mod_down2;
  bool has_rescale = false;
  int restore_start = 0, restore_end = 0;
  std::vector<u64> rs1, rs_inv, rs_pad, mdr1, mdr_inv, mdr_pad;
  std::vector<i64> rs2, mdr2;
  std::vector<i64 *> d_mod_up2;
  i64 *d_mod_down2 = nullptr, *d_rs2 = nullptr, *d_mdr2 = nullptr;
};
void build_level_ms64(const Params64 &P, int level, LevelMS64 *m);

struct Ct64 {
  NP np;
  double scale = 1.0;
  int num_slots = 0;
  bool has_rx = false;  // the third part of an unrelinearised product
  u64 *bx = nullptr, *ax = nullptr, *rx = nullptr;
  size_t cap_words = 0, rx_cap_words = 0;
  Ct64() = default;
  Ct64(const Ct64 &) = delete;
  Ct64 &operator=(const Ct64 &) = delete;
  ~Ct64();
  // capacity for np (and an rx part when rx); keeps the words already there
  // only when no buffer grows
  Status reserve(const NP &np, int n, bool rx = false);
  void swap(Ct64 &o);
};

struct Evk64 {
  NP np;  // key basis (max level + aux)
  int beta = 0;
  u64 *bx = nullptr, *ax = nullptr;  // [beta][np.total()][N]
  ~Evk64();
};

class Context64 {
 public:
  ~Context64();
  Status init(const ParamSpec64 &spec, int dev, std::string *err);
  std::unique_ptr<Params64> P;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  // scratch of the operations: a stack of device chunks reused across calls
  // (every operation runs on the context stream, so a later call's scratch
  // may reuse an earlier call's words)
  Arena arena;
  u64 *d_primes = nullptr;
  i64 *d_qinv = nullptr;
  ulonglong2 *d_tw = nullptr, *d_itw = nullptr;  // [nprimes][N] (w, floor(w 2^64 / q))
  std::vector<u64> n_inv, mont_conv, r_inv, n_inv_mont_inv;
  std::vector<u64> p_prod;  // Montgomery P mod q_i for the q primes of the key basis
  std::vector<std::unique_ptr<LevelMS64>> ms;  // index level + 1
  const LevelMS64 &lms(int level);
  const ulonglong2 *tw(int g) const { return d_tw + (static_cast<size_t>(g) << P->log_n); }
  const ulonglong2 *itw(int g) const { return d_itw + (static_cast<size_t>(g) << P->log_n); }
  void shoup(u64 c, int g, u64 *w, u64 *ws) const;       // plain constant c
  void mont_shoup(u64 c, int g, u64 *w, u64 *ws) const;  // c R^-1: multiplies a Montgomery value by c
  Status check(const char *where);

  // raw transforms of `count` polynomials over np's primes, in place
  Status ntt(const NP &np, u64 *data, int count, bool mont);
  Status intt(const NP &np, u64 *data, int count, bool mont);
  // ModUp of src [q][N] into beta outputs dst + i [tot][N]
  Status modup(int level, const u64 *src, u64 *dst);
  // ModDown family of npoly polynomials
  Status moddown(int level, MDType type, const u64 *const *src, u64 *const *dst, int npoly);
  // evaluator
  Status hmult(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key, bool rescale);
  Status hrot(Ct64 &res, const Ct64 &a, const Evk64 &key, int rot);
  Status hconj(Ct64 &res, const Ct64 &a, const Evk64 &key);
  Status key_switch_permute(Ct64 &res, const Ct64 &a, const Evk64 &key, u64 galois);
  Status rescale(Ct64 &res, const Ct64 &a);
  // Context<uint64_t> operations (Context.cpp:101-949): element-wise
  // arithmetic, the three-part tensor, relinearisation, key switching
  // without the automorphism, automorphisms, level-down
  Status copy(Ct64 &res, const Ct64 &a);
  Status add(Ct64 &res, const Ct64 &a, const Ct64 &b);
  Status sub(Ct64 &res, const Ct64 &a, const Ct64 &b);
  Status neg(Ct64 &res, const Ct64 &a);
  Status mult_tensor(Ct64 &res, const Ct64 &a, const Ct64 &b);
  Status relinearize(Ct64 &res, const Ct64 &a, const Evk64 &key, bool rescale);
  Status mult_key(Ct64 &res, const Ct64 &a, const Evk64 &key);
  Status permute(Ct64 &res, const Ct64 &a, int rot, bool conjugate);
  Status hrot_add(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key, int rot);
  Status hconj_add(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key);
  Status mult_imag_unit(Ct64 &res, const Ct64 &a);
  // constants: one Montgomery word per prime of the operand's basis
  Status mult_const(Ct64 &res, const Ct64 &a, const u64 *cx, double cscale);
  Status add_const(Ct64 &res, const Ct64 &a, const u64 *cx);
  Status level_down(Ct64 &res, const Ct64 &a, int target_level);
  // Encoder::EncodeConstant (Encode.cpp:250-275) with 64-bit words
  void encode_const(int level, double scale, double value, int num_aux, std::vector<u64> *cx) const;
  std::vector<u64> imag_unit;  // psi^(N/2) per prime, Montgomery
  // key switch of d (q primes, NTT domain) with key, plus P (d0, d1) on the
  // q rows (either may be null): acc (b, a) over Q u P
  Status key_mult(int level, const u64 *d, const u64 *d0, const u64 *d1, const Evk64 &key, u64 *acc_b, u64 *acc_a);
};

}  // namespace w64
}  // namespace chd

// ---- kernels (w64_kernels.cu) ---------------------------------------------
namespace chd {
namespace w64 {

// One limb of a batched transform; constants are plain residues with their
// Shoup companions floor(w 2^64 / q).  Flags as RowFlags of the 32-bit path.
struct Row64 {
  const u64 *src;
  u64 *dst;
  const u64 *src2;
  const ulonglong2 *tw;
  u64 q;
  i64 qinv;
  uint32_t flags, pad_;
  u64 c0, c0s, c1, c1s, c2, c2s;
};
constexpr int kMaxRows64 = 64;
struct RowBatch64 {
  int count;
  Row64 rows[kMaxRows64];
};
// forward: column phase then row phase (N = 2^16), in place allowed
void launch_ntt64_fwd(const RowBatch64 &rb, cudaStream_t s);
// inverse: row phase then column phase, output x c0 (canonical or centred)
void launch_ntt64_inv(const RowBatch64 &rb, cudaStream_t s);

// out[m][n] = REDC(sum_k xt[k][n] T[m][k]) mod p_m (xt centred, T centred)
struct BConv64Job {
  const i64 *xt;
  u64 *out;
  const i64 *table;  // device [M][K]
  int K, M;
  uint8_t out_row[64], out_gidx[64];
};
constexpr int kMaxBConv64Jobs = 16;
struct BConv64Batch {
  int count;
  const u64 *primes;
  const i64 *qinvs;
  BConv64Job jobs[kMaxBConv64Jobs];
};
void launch_bconv64(const BConv64Batch &b, cudaStream_t s);

// per-limb element-wise kernels
struct Elem64Row {
  const u64 *a1, *b1, *a2, *b2;  // operands (meaning per op)
  u64 *o0, *o1, *o2;
  u64 q;
  i64 qinv;
  u64 c;  // per-row constant (Elem64Op)
};
constexpr int kMaxElem64Rows = 64;
struct Elem64Batch {
  int count;
  Elem64Row rows[kMaxElem64Rows];
};
// tensor: o0 = b1 b2, o1 = b1 a2 + a1 b2, o2 = a1 a2 (Montgomery products)
void launch_tensor64(const Elem64Batch &b, cudaStream_t s);
// o0 = a1 + b1 (mod q)
void launch_add64(const Elem64Batch &b, cudaStream_t s);
// o0 = op(a1[, b1 | c]) on canonical residues; kMult and kMultConst are
// Montgomery products, kMultImagUnit multiplies by c in the first half of
// the evaluation domain and by -c in the second (X^(N/2))
enum class Elem64Op { kAdd, kSub, kNeg, kMult, kMultConst, kAddConst, kCopy, kMultImagUnit };
void launch_elem64(Elem64Op op, const Elem64Batch &b, cudaStream_t s);
// o0[k] = a1[galois(k)] (the automorphism in the bit-reversed domain)
void launch_permute64(const Elem64Batch &b, u64 galois, cudaStream_t s);

// key inner product of one row r of the extended basis:
// acc_b = sum_i mu_i kb_i (+ p d0), acc_a = sum_i mu_i ka_i (+ p d1)
struct KeyMac64Row {
  const u64 *mu[8];
  const u64 *kb[8], *ka[8];
  const u64 *d0, *d1;  // nullptr on aux rows
  u64 *acc_b, *acc_a;
  u64 q, p;            // p: Montgomery P mod q
  i64 qinv;
  int beta;
};
constexpr int kMaxKeyMac64Rows = 16;
struct KeyMac64Batch {
  int count;
  KeyMac64Row rows[kMaxKeyMac64Rows];
};
void launch_key_mac64(const KeyMac64Batch &b, cudaStream_t s);

}  // namespace w64
}  // namespace chd
