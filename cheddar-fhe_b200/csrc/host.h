// Host-side model of the CKKS evaluation core: parameter / level model,
// per-level ModSwitch constants, device tables, device ciphertexts and keys,
// and the evaluator that composes the CUDA kernels.  The public C ABI
// (include/cheddar_b200.h) is a thin layer over this.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <complex>
#include <functional>
#include <vector>

#include "kernels.h"

namespace chd {

// ---- errors ----------------------------------------------------------------
enum Status : int {
  kOk = 0,
  kErrInvalidArg = 1,
  kErrInvalidLevel = 2,
  kErrShape = 3,
  kErrCuda = 4,
  kErrAlloc = 5,
  kErrUnsupported = 6,
  kErrKey = 7,
  kErrParse = 8,
};
void set_error(const std::string &msg);
const char *last_error();

struct Error {
  Status code;
  std::string msg;
};

// ---- prime utilities ---------------------------------------------------------
namespace prime {
uint32_t mul_mod(uint32_t a, uint32_t b, uint32_t q);
uint32_t pow_mod(uint32_t a, int64_t e, uint32_t q);
uint32_t inv_mod(uint32_t a, uint32_t q);
uint32_t smallest_generator(uint32_t q);
uint32_t primitive_root(uint32_t m, uint32_t q);
int32_t inv_mod_word(uint32_t q);
uint32_t to_mont(uint32_t a, uint32_t q);
int32_t centre(uint32_t a, uint32_t q);
}  // namespace prime

// ---- level model -------------------------------------------------------------
struct NP {
  int main = 0, ter = 0, aux = 0;
  int q() const { return main + ter; }
  int total() const { return main + ter + aux; }
  bool operator==(const NP &o) const { return main == o.main && ter == o.ter && aux == o.aux; }
};

// The reference's Parameter fields for word size W (uint32_t, or uint64_t
// for the 64-bit word path).
template <typename W>
struct ParamSpecT {
  int log_degree = 16;
  double base_scale = 0;
  int default_encryption_level = 0;
  std::vector<std::pair<int, int>> level_config;
  std::vector<W> main_primes, aux_primes, ter_primes;
  std::pair<int, int> additional_base{0, 0};
  int dense_hw = -1, sparse_hw = 32;
  bool boot = false;
  int num_cts_levels = 0, num_stc_levels = 0;
};
using ParamSpec = ParamSpecT<uint32_t>;
using ParamSpec64 = ParamSpecT<uint64_t>;

// Parses the reference's parameter JSON schema (primes read as exact
// integers; a prime beyond the word is kept as the word's maximum, which
// validation rejects).
bool parse_param_json(const std::string &text, ParamSpec *out, std::string *err);
bool parse_param_json64(const std::string &text, ParamSpec64 *out, std::string *err);

class Params {
 public:
  static std::unique_ptr<Params> create(const ParamSpec &spec, std::string *err);

  ParamSpec spec;
  int log_n = 0, n = 0, L = 0, alpha = 0, max_ter = 0, max_main = 0, max_level = 0;
  NP short_np;                   // level -1 base
  std::vector<uint32_t> primes;  // global order: ter reversed, main, aux
  std::vector<int32_t> qinv;
  std::vector<int> galois;       // 5^i mod 2N, i in [0, N/2]
  std::vector<double> scale, rescale_prod;

  NP level_np(int level, int num_aux = 0) const;
  int np_to_level(const NP &np) const;  // -2 if not a level
  void gidx(const NP &np, int *out) const;
  int sse_num_aux() const;
  uint32_t galois_of(int amount) const;  // amount in [0, N/2] or -1
};

// Per-level ModSwitch constants (host and device copies).
struct LevelMS {
  int level = 0, num_aux = 0, beta = 0, num_q = 0;
  std::vector<uint32_t> mod_up1;
  std::vector<int> dig_s, dig_e;
  std::vector<std::vector<int32_t>> mod_up2;  // host [dst][src] per digit
  std::vector<uint32_t> mod_down1, inv_p_prod;
  std::vector<int32_t> mod_down2;
  bool has_rescale = false;
  int pad_start = 0, pad_end = 0, restore_start = 0, restore_end = 0;
  int rs_src_len = 0, mdr_src_len = 0, rs_dst_len = 0;
  std::vector<uint32_t> rs1, rs_inv, rs_pad, mdr1, mdr_inv, mdr_pad;
  std::vector<int32_t> rs2, mdr2;
  // device copies of the BConv tables
  std::vector<int32_t *> d_mod_up2;
  int32_t *d_mod_down2 = nullptr, *d_rs2 = nullptr, *d_mdr2 = nullptr;
};

// Host-only computation of the ModSwitch constants of one level (no GPU).
void build_level_ms(const Params &P, int level, LevelMS *m);

// ---- device objects ----------------------------------------------------------
struct DeviceCt {
  NP np;
  bool has_rx = false;
  double scale = 1.0;
  int num_slots = 0;
  uint32_t *bx = nullptr, *ax = nullptr, *rx = nullptr;
  size_t cap_words = 0;  // allocated words per part
  bool owned = true;
  DeviceCt() = default;
  DeviceCt(const DeviceCt &) = delete;
  DeviceCt &operator=(const DeviceCt &) = delete;
  // moves transfer the buffers (containers of ciphertexts may reallocate)
  DeviceCt(DeviceCt &&o) noexcept { take(o); }
  DeviceCt &operator=(DeviceCt &&o) noexcept;
  ~DeviceCt();
  Status reserve(const NP &np, bool rx, int n);

 private:
  void take(DeviceCt &o) noexcept {
    np = o.np;
    has_rx = o.has_rx;
    scale = o.scale;
    num_slots = o.num_slots;
    bx = o.bx;
    ax = o.ax;
    rx = o.rx;
    cap_words = o.cap_words;
    owned = o.owned;
    o.bx = o.ax = o.rx = nullptr;
    o.cap_words = 0;
  }
};

struct DeviceEvk {
  int beta = 0;
  NP np;  // key basis (all q primes + alpha aux primes)
  uint32_t *bx = nullptr, *ax = nullptr;  // [beta][np.total][N]
  bool owned = true;
  ~DeviceEvk();
};

// Stack arena over device memory: chunks are never moved, so pointers handed
// out during an operation stay valid until the matching release.
class Arena {
 public:
  ~Arena();
  void *alloc(size_t bytes);
  size_t mark() const { return top_; }
  void release(size_t m);

 private:
  struct Chunk {
    char *p;
    size_t size;
    size_t start;  // global offset of this chunk
  };
  std::vector<Chunk> chunks_;
  size_t top_ = 0;   // global offset
  size_t total_ = 0;
};

// Error helpers of the host code: record the message, return the status.
#define CHD_CHECK(cond, code, msg) \
  do {                             \
    if (!(cond)) {                 \
      set_error(msg);              \
      return code;                 \
    }                              \
  } while (0)
#define CHD_TRY(expr)            \
  do {                           \
    Status _s = (expr);          \
    if (_s != kOk) return _s;    \
  } while (0)

// Square complex matrix stored by diagonals: d[i][k] = M[k][(k + i) mod w]
// (StripedMatrix, include/extension/StripedMatrix.h).
struct SMat {
  int h = 0, w = 0;
  std::map<int, std::vector<std::complex<double>>> d;
};
SMat smat_mult(const SMat &a, const SMat &b);
SMat smat_scale(const SMat &a, std::complex<double> b);

// A compiled linear transform (LinearTransform + HoistHandler): encoded
// diagonals keyed by (giant step, baby step), device plaintexts over the
// Q u P basis of pt_level.
struct LTPlan {
  struct Pt {
    int gs = 0, bs = 0;
    std::vector<std::complex<double>> msg;
    uint32_t *dev = nullptr;
  };
  int pt_level = 0, width = 0, pt_slots = 0;
  double pt_scale = 0;
  std::vector<int> bs_idx, gs_idx;  // sorted
  std::vector<Pt> pts;              // giant step major, baby step minor
  LTPlan() = default;
  LTPlan(const LTPlan &) = delete;
  LTPlan &operator=(const LTPlan &) = delete;
  LTPlan(LTPlan &&) = default;
  LTPlan &operator=(LTPlan &&) = default;
  ~LTPlan();
};
struct DeviceEvk;
using RotKeys = std::map<int, const DeviceEvk *>;
// The keys a program may use (EvkMap: multiplication, conjugation,
// rotations, and the dense-to-sparse / sparse-to-dense keys of
// sparse-secret encapsulation)
struct ProgKeys {
  const DeviceEvk *mult = nullptr, *conj = nullptr, *dts = nullptr, *std_key = nullptr;
  const RotKeys *rot = nullptr;
  bool min_ks = false;  // linear transforms in the min-KS form
};

// A straight-line program of ciphertext operations over registers, the
// compiled form of EvalPoly / EvalMod / Boot (planning on the host, every
// op a call of the device evaluator).  Constants are (level, scale, value)
// triples encoded with Encoder::EncodeConstant.
struct ProgConst {
  int level = 0;
  double scale = 1.0, value = 0.0;
};
enum class OpKind : int {
  kConstMult = 0,   // dst = a (.) c at `level`               (Context::MultUnsafe Ct x Const)
  kTensor = 1,      // dst = a x b at `level`, three parts       (Context::MultUnsafe Ct x Ct)
  kConstAccum = 2,  // dst = sum_i src_i (.) c_i (+ plain) at `level` (ElementWiseHandler::CAccum)
  kAddConst = 3,    // dst = a + c (b part)                      (Context::Add Ct + Const)
  kAdd = 4,         // dst = a + b                               (Context::Add Ct + Ct)
  kRelinRescale = 5,// dst = RelinearizeRescale(a)
  kRescale = 6,     // dst = Rescale(a)
  kLevelDown = 7,   // dst = Rescale(a (.) c), c = 1 at the rescale prime product (AddLowerLevelsUntil)
  kCopy = 8,
  kSetScale = 9,    // metadata only
  kSub = 10,        // dst = a - b
  kHConj = 11,      // dst = HConj(a)
  kMultImag = 12,   // dst = i * a
  kModUpToMax = 13, // dst = ModUpToMax(a)
  kHRotAdd = 14,    // dst = HRot(a, r) + b
  kLinTrans = 15,   // dst = lin_trans[lt](a)
  kSetSlots = 16,   // metadata only: dst.num_slots = rot
};
struct ProgOp {
  OpKind kind = OpKind::kCopy;
  int dst = -1, a = -1, b = -1;
  int level = 0;
  int c = -1;                   // constant index
  std::vector<int> srcs, cs;    // kConstAccum terms
  int plain = -1;               // kConstAccum plain addend (may be dst itself)
  int rot = 0;                  // kHRotAdd rotation, kLinTrans transform index
  double scale = 0.0;           // kSetScale
};
struct Program {
  int nregs = 0, input = 0, output = 0;
  std::vector<ProgConst> consts;
  std::vector<ProgOp> ops;
  int add_const(int level, double scale, double value) {
    consts.push_back(ProgConst{level, scale, value});
    return static_cast<int>(consts.size()) - 1;
  }
  int reg() { return nregs++; }
};

// A prepared bootstrapping (BootContext + EvalSpecialFFT + EvalMod for one
// slot count): the CtS then StC linear transforms and the Boot program.
struct BootPlan {
  int num_slots = 0, max_level = 0, cts_start = 0, em_start = 0, stc_start = 0, end_level = 0, log_scaleup = 0;
  int variant = 0;  // BootVariant: 0 kNormal, 1 kImaginaryRemoving, 2 kMergeTwoReal
  double cts_const = 0, stc_const = 0, em_start_scale = 0, em_end_scale = 0, final_scale = 0;
  std::vector<LTPlan> lts;
  std::vector<const LTPlan *> lt_ptrs;
  Program prog;
  std::vector<int> rotations;  // rotation keys the transforms use
  std::vector<int> extra_rotations;  // sparse slots: Trace and the last StC fold
};

// EvalMod cosine polynomial of the reference's BootParameter
const std::vector<double> &boot_mod_coefficients();

// HoistHandler::CheckStrideMinKS: the baby / giant strides of a plan
Status lt_min_ks_strides(const LTPlan &pl, int *bs_stride, int *gs_stride);

// Exchanges two ciphertexts' buffers and metadata
void swap_regs(DeviceCt &x, DeviceCt &y);

// A ciphertext whose buffers come from the arena (not owned; released with
// the enclosing ArenaScope)
Status scratch_ct(Arena &arena, DeviceCt &t, const NP &np, bool rx, int n);

// Releases everything allocated from the arena inside a scope.
struct ArenaScope {
  Arena &a;
  size_t m;
  explicit ArenaScope(Arena &x) : a(x), m(x.mark()) {}
  ~ArenaScope() { a.release(m); }
};
// The same, or (hold) leaves the allocations to the enclosing scope.
struct HeldScope {
  Arena &a;
  size_t m;
  bool hold;
  HeldScope(Arena &x, bool h) : a(x), m(x.mark()), hold(h) {}
  ~HeldScope() {
    if (!hold) a.release(m);
  }
};

class Context {
 public:
  static std::unique_ptr<Context> create(const ParamSpec &spec, int device, std::string *err);
  ~Context();

  std::unique_ptr<Params> P;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Arena arena;

  // device tables
  uint32_t *d_primes = nullptr;
  int32_t *d_qinv = nullptr;
  int *d_err = nullptr;   // set by kernels whose bounded waits ran out
  // test hook (chd_debug_stall_tensor_waits): > 0 makes the stand-alone
  // tensor-core base conversion's bounded waits run out
  uint32_t tc_stall_polls = 0;
  int num_sms = 0;
  int ks_engine = 0;      // ModUp / ModDown column-pass base conversion: 0 CUDA cores, 1 tensor cores, 2 autotuned
  // A fused key switch of two or more ciphertexts runs its two halves on the
  // context stream and on aux_stream (forked from and joined back into the
  // context stream by events), so that the kernels of one half fill the
  // issue slots the other half's kernels leave idle (the column passes wait
  // on barriers and the tensor cores, the row passes on the ALU)
  bool split_streams = true;
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  uint2 *d_tw = nullptr, *d_itw = nullptr;  // [nprimes][N] (psi_rev, Shoup companion)
  std::vector<uint32_t> n_inv, n_inv_mont, mont_conv, p_prod, imag_unit;
  std::vector<uint32_t> r_inv;  // 2^-32 mod q per global prime
  std::vector<LevelMS> ms;  // index level + 1
  std::vector<std::complex<double>> enc_tw;  // e^(2 pi i k / 2N), built on first use
  const std::vector<std::complex<double>> &enc_twiddles();

  const LevelMS &lms(int level) const { return ms.at(level + 1); }
  const uint2 *tw(int g) const { return d_tw + (static_cast<size_t>(g) << P->log_n); }
  const uint2 *itw(int g) const { return d_itw + (static_cast<size_t>(g) << P->log_n); }
  // (w, companion) that multiplies like a Montgomery product by c: c 2^-32 mod q
  void mont_as_shoup(uint32_t c, int g, uint32_t *w, uint32_t *ws) const;

  // ---- building blocks on raw device pointers ----
  // NTT of the limbs of np stored contiguously at data (in place)
  Status ntt(const NP &np, uint32_t *data, bool mont, int count = 1, size_t stride = 0);
  Status intt(const NP &np, uint32_t *data, bool mont, int count = 1, size_t stride = 0);
  // ModUp of src [num_q][N] at `level` into dst[beta] ([num_q + aux][N] each)
  Status modup(int level, const uint32_t *src, uint32_t *const *dst);
  Status modup_many(int level, int count, const uint32_t *const *src, uint32_t *const *const *dst);
  Status modup_fused(int level, int count, const uint32_t *const *src, uint32_t *const *const *dst,
                     uint32_t *rows_out);
  enum class MDType { kModDown, kRescale, kModDownRescale };
  // Which rows a ModDown / Rescale / ModDownAndRescale drops and the
  // constants of its BConv and epilogue (ModSwitch.cu:566-684).
  struct MDPlan {
    NP ns, nd, nn;
    int src_len = 0, dst_len = 0, src2_start = 0, src2_end = 0, src2_off = 0;
    std::vector<int> srows, gs, gd;
    const uint32_t *c1 = nullptr, *inv = nullptr, *pad = nullptr;
    const int32_t *table = nullptr;
  };
  Status moddown_plan(int level, MDType type, MDPlan *plan) const;
  // Fused N = 2^16 key switch (see keyswitch.cu): count inputs at one level,
  // results written to out_b / out_a after ModDown (or ModDownAndRescale).
  struct KSIn {
    int mode;  // 0 HMult (b1,a1,b2,a2), 1 MultKey (b1=bx, a1=ax), 2 Relinearize (b1=bx, a1=ax, a2=rx)
    const uint32_t *b1, *a1, *b2, *a2;
    uint32_t *out_b, *out_a;
  };
  // INTT rows -> ModUp column pass -> key-switch row pass -> ModDown column
  // pass -> NTT rows with the ModDown epilogue, for `count` inputs.  With
  // keep_ext the pipeline stops after the row pass: out_b / out_a receive the
  // accumulators over every prime of Q u P (evaluation domain), `type` is
  // unused, and mode 1 with b1 == nullptr leaves out the P * bx term (the
  // bare inner product sum_i ModUp(a1)_i (.) key_i).
  Status key_switch_fused(int level, int count, const KSIn *in, const DeviceEvk &key, MDType type,
                          bool keep_ext = false);
  // The same pipeline with ciphertext c at levels[c]: every stage is one
  // launch (or a few, by the per-launch job limits) over all levels.
  Status key_switch_fused_levels(const int *levels, int count, const KSIn *in, const DeviceEvk &key, MDType type,
                                 bool keep_ext = false);
  // one pipeline on the context stream; with hold the scratch stays
  // allocated in the caller's arena scope
  Status key_switch_fused_pipeline(const int *levels, int count, const KSIn *in, const DeviceEvk &key, MDType type,
                                   bool keep_ext, bool hold);
  // ModDown family on npoly polys
  Status moddown(int level, MDType type, const uint32_t *const *src, uint32_t *const *dst, int npoly);
  // one ModDown pipeline on the context stream (hold: as in
  // key_switch_fused_pipeline)
  Status moddown_pipeline(int level, MDType type, const uint32_t *const *src, uint32_t *const *dst, int npoly,
                          bool hold);
  // half(false) on the context stream, then half(true) on aux_stream,
  // forked from and joined back into the context stream; both halves'
  // arena scratch lives until the join is enqueued
  Status fork_halves(const std::function<Status(bool)> &half);
  // launch(batch, stream) per batch of for_row_batches, alternating between
  // the context stream and aux_stream when there are several batches of
  // disjoint rows
  Status alternate_row_batches(const std::vector<RowDesc> &rows, bool disjoint,
                               const std::function<void(const RowBatch &, cudaStream_t)> &launch, const char *what);
  Status bconv(const int32_t *xt, int K, const int32_t *table, const int *dst_gidx, int M, uint32_t *out);
  // BConv of npoly polynomials ([npoly][K][N] -> [npoly][M][N]) with the
  // host table T[m][k] (centred, Montgomery q-hat R^2): engine 0 on the CUDA
  // cores (int64 multiply-adds), engine 1 on the tcgen05 tensor cores (INT8
  // limb split); identical results.
  Status bconv_many(int engine, int npoly, const int32_t *xt, int K, const std::vector<int32_t> &table,
                    const int *dst_gidx, int M, uint32_t *out);

  // ---- evaluator (Context.cpp of the reference) ----
  Status add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b);
  Status sub(DeviceCt &res, const DeviceCt &a, const DeviceCt &b);
  Status neg(DeviceCt &res, const DeviceCt &a);
  Status mult_tensor(DeviceCt &res, const DeviceCt &a, const DeviceCt &b);
  Status mult_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, double cscale);
  Status add_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx);
  Status mult_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt_dev, double pscale);
  Status mult_imag_unit(DeviceCt &res, const DeviceCt &a);
  Status rescale(DeviceCt &res, const DeviceCt &a);
  Status relinearize(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key, bool rescale);
  Status hmult(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key, bool rescale);
  Status hmult_batch(int count, DeviceCt *const *res, const DeviceCt *const *a, const DeviceCt *const *b,
                     const DeviceEvk &key, bool rescale);
  Status mult_key(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key);
  Status permute(DeviceCt &res, const DeviceCt &a, int amount);
  Status hrot(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key, int dist);
  Status hconj(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key);
  Status hrot_add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key, int dist);
  // hoisted baby-step rotations, outputs stay in the Q u P basis
  Status hoisted_rotate(const DeviceCt &a, int R, const int *dists, const DeviceEvk *const *keys,
                        DeviceCt *const *out);
  // the same rotations of `count` ciphertexts at one level: one batched
  // ModUp, keys read once per launch for up to kMaxHoistCts ciphertexts;
  // out[c][j] is rotation j of ciphertext c
  Status hoisted_rotate_batch(int count, const DeviceCt *const *a, int R, const int *dists,
                              const DeviceEvk *const *keys, DeviceCt *const *const *out);
  // ModDown of a Q u P ciphertext back to Q
  Status moddown_ct(DeviceCt &res, const DeviceCt &a);
  Status moddown_batch(int count, DeviceCt *const *res, const DeviceCt *const *a);

  // ---- bootstrapping building blocks (boot.cu) ----
  // Encoder::Encode (Encode.cpp:23-41, 84-107, 135-190): msg_len complex
  // slots (padded to a power of two) -> plaintext [level_np(level, num_aux)]
  // in the NTT Montgomery domain at pt_dev; waits for the upload.
  Status encode(int level, double scale, const std::complex<double> *msg, int msg_len, int num_aux,
                uint32_t *pt_dev, int *num_slots_out);
  // Encoder::EncodeConstant (Encode.cpp:250-275): Montgomery residues
  void encode_const(int level, double scale, double value, int num_aux, std::vector<uint32_t> *cx) const;
  // Encoder::Decode (Encode.cpp:45-70, 109-133, 192-248): plaintext at
  // `level` (no aux primes, NTT Montgomery domain) -> num_slots complex
  // slots (a power of two <= N/2) at out; waits for the result.
  Status decode(int level, double scale, const uint32_t *pt_dev, int num_slots, std::complex<double> *out);
  // device copies of the encoder's twiddles e^(2 pi i k / 2N) and 5^i mod 2N
  double2 *d_enc_tw = nullptr;
  int *d_galois = nullptr;
  Status codec_tables();
  // BootContext::ModUpToMax without sparse-secret encapsulation
  // (BootContext.cpp:186-270): level -1 -> top level
  Status modup_to_max(DeviceCt &res, const DeviceCt &a);
  // ... with sparse-secret encapsulation: dense-to-sparse key switch at level
  // -1, lift, single-digit sparse-to-dense key switch, ModDown
  Status modup_to_max_sse(DeviceCt &res, const DeviceCt &a, const DeviceEvk &dts, const DeviceEvk &std_key);
  // Parameter::IsUsingSparseSecretEncapsulation (Parameter.cu:246-248),
  // with the reference's default dense Hamming weight N/2 (Parameter.cu:40)
  int dense_hw() const { return P->spec.dense_hw > 0 ? P->spec.dense_hw : P->n / 2; }
  bool uses_sse() const { return dense_hw() > P->spec.sparse_hw; }

  // Linear transform planning and evaluation (lintrans.cu): LinearTransform
  // ctor + HoistHandler ctor (LinearTransform.cpp:8-75, Hoist.cu:120-167)
  Status lt_build(const SMat &m, int pt_level, double pt_scale, int bs, int gs, int pre_rotation,
                  int additional_pt_rot, bool suppress_swap, LTPlan *out);
  // HoistHandler::Evaluate (Hoist.cu:554-975): res at pt_level - 1
  Status lt_evaluate(DeviceCt &res, const DeviceCt &in, const LTPlan &pl, const RotKeys &keys);
  // the same transform on `count` ciphertexts at one level, launches batched
  Status lt_evaluate_batch(int count, DeviceCt *const *res, const DeviceCt *const *in, const LTPlan &pl,
                           const RotKeys &keys);
  // the min-KS evaluation (Hoist.cu:490-552): two rotation keys per transform
  Status lt_evaluate_min_ks(DeviceCt &res, const DeviceCt &in, const LTPlan &pl, const RotKeys &keys);
  Status lt_evaluate_min_ks_batch(int count, DeviceCt *const *res, const DeviceCt *const *in, const LTPlan &pl,
                                  const RotKeys &keys);
  // HRot (dist >= 0) or HConj (dist = -1) of `count` ciphertexts at one
  // level with one key: a single fused key switch over the batch, then the
  // automorphisms; res[c] may alias a[c]
  Status hrot_batch(int count, DeviceCt *const *res, const DeviceCt *const *a, const DeviceEvk &key, int dist);

  // EvalPoly::Compile (EvalPoly.cpp:750-830) of a polynomial in the
  // Chebyshev (or power) basis for an input at (input_level, input_scale):
  // appends the evaluation to `prog` reading register `in`, returns the
  // result register (scale target_scale, level input_level - ceil(log2(deg+1))).
  Status compile_poly(Program &prog, int in, const std::vector<double> &coeffs, int input_level, double input_scale,
                      double target_scale, bool chebyshev, int *out_reg, int *out_level);
  // EvalMod (EvalMod.cpp:9-61): x -> mod-reduction approximation, appended to prog
  Status compile_evalmod(Program &prog, int in, int start_level, const std::vector<double> &mod_coeffs,
                         int num_double_angle, int initial_K, int *out_reg, int *out_level, double *start_scale,
                         double *end_scale);
  // Runs a program (program.cu): regs[input] holds the input
  Status run_program(const Program &prog, std::vector<DeviceCt> &regs, const ProgKeys &keys,
                     const std::vector<const LTPlan *> *lts);
  // the program on `count` ciphertexts (registers R[c]); key switches,
  // rescales and linear transforms batched across them
  Status run_program_batch(const Program &prog, int count, std::vector<DeviceCt> *const *R, const ProgKeys &keys,
                           const std::vector<const LTPlan *> *lts);
  bool mult_unsafe_compatible(int l1, int l2) const;
  // the remaining public Context operations (ops_ext.cu)
  Status copy_ct(DeviceCt &res, const DeviceCt &a);
  Status mult_unsafe(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, int level);
  Status mult_unsafe_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, int const_level, double const_scale,
                           int level);
  Status mad_unsafe(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, int const_level, double const_scale);
  Status permute_ct(DeviceCt &res, const DeviceCt &a, int rot_dist, bool conjugate);
  Status hconj_add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key);
  Status level_down(DeviceCt &res, const DeviceCt &a, int target_level);
  Status mult_key_no_moddown(DeviceCt &accum, const DeviceCt &a, const DeviceEvk &key);
  Status add_sub_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt, double pscale, bool subtract);
  Status sub_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx);
  Status sub_from(DeviceCt &res, const uint32_t *pt, const uint32_t *cx, double scale, const DeviceCt &b);
  Status mult_unsafe_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt, int pt_level, int pt_aux,
                           double pscale, int level);
  // sizes the registers of a program (plus two spares) at top-level capacity
  Status program_regs(const Program &prog, std::vector<DeviceCt> &regs);
  // BootContext (bootplan.cu): prepare full-slot bootstrapping with
  // num_cts / num_stc levels for CoeffToSlot / SlotToCoeff
  Status boot_build(int num_slots, int variant, int num_cts, int num_stc, int log_msg_ratio, BootPlan *out);
  // BootContext::Boot: in at level 0 -> res at the end level.  regs_io,
  // when given, keeps the program registers allocated across calls.
  Status boot_run(const BootPlan &bp, DeviceCt &res, const DeviceCt &in, const ProgKeys &keys,
                  std::vector<DeviceCt> *regs_io);
  // Boot of `count` ciphertexts (each with its own program registers),
  // key switches, rescales and linear transforms batched across them
  Status boot_run_batch(const BootPlan &bp, int count, DeviceCt *const *res, const DeviceCt *const *in,
                        const ProgKeys &keys, std::vector<DeviceCt> *const *regs);

  // ---- optional device timing of the fused key-switch stages ----
  // Events recorded on the context stream around each stage's launches.
  enum KsStage { kKsInvRows, kKsModUpCols, kKsRows, kKsModDownCols, kKsFwdRows, kKsStages };
  struct StageTimer {
    bool on = false;
    std::vector<cudaEvent_t> ev;  // pool, reused across sessions
    int used = 0;
    struct Span {
      int stage, e0, e1, launches;
    };
    std::vector<Span> spans;
  } timer;
  int timer_mark();                                   // records an event; -1 when off
  void timer_span(int stage, int e0, int launches);   // closes a span opened by timer_mark
  Status timer_read(double *ms, int *launches);       // sums per stage (waits for the stream)

 private:
  Status init(const ParamSpec &spec, int dev, std::string *err);
  Status check_cuda(const char *where);
  // key-switch core: accum = sum_i ModUp(d_in)_i (.) key_i (+ P*(d0,d1))
  struct KSJob {
    const uint32_t *d0, *d1, *d_in;
    uint32_t *acc_b, *acc_a;
  };
  Status key_switch_core(int level, const uint32_t *d0, const uint32_t *d1, const uint32_t *d_in,
                         const DeviceEvk &key, uint32_t *acc_b, uint32_t *acc_a);
  Status key_switch_many(int level, int count, const KSJob *jobs, const DeviceEvk &key);
};

// one element-wise op over `parts` parts of every row of np (row r of part
// p at dst[p] + r * N, likewise a / b), per-row constant k[r]
Status elem_parts(Context &C, ElemOp op, const NP &np, int parts, uint32_t *const *dst, const uint32_t *const *a,
                  const uint32_t *const *b, const uint32_t *k);

// Splits a long list of rows into RowBatch launches: as few launches as
// `cap` rows per launch (at most kMaxRows) allow, with the rows spread
// evenly over them (a short last launch would leave most SMs idle).
template <typename F>
void for_row_batches(const std::vector<RowDesc> &rows, F &&launch, int cap = kMaxRows) {
  cap = cap < 1 || cap > kMaxRows ? kMaxRows : cap;
  const int total = static_cast<int>(rows.size());
  const int nbat = (total + cap - 1) / cap;
  const int per = nbat > 0 ? (total + nbat - 1) / nbat : cap;
  RowBatch rb;
  rb.count = 0;
  for (const RowDesc &r : rows) {
    rb.rows[rb.count++] = r;
    if (rb.count == per) {
      launch(rb);
      rb.count = 0;
    }
  }
  if (rb.count) launch(rb);
}

// Makes `device` current for the scope of a C ABI call and restores the
// caller's device afterwards: kernels, allocations and stream work of a
// context always run on the device it was created on, whichever device the
// calling thread has current.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device) changed_ = cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (changed_) cudaSetDevice(prev_);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;

 private:
  int prev_ = -1;
  bool changed_ = false;
};

}  // namespace chd

// The C ABI's opaque handles (include/cheddar_b200.h) that more than one
// translation unit implementing entry points uses.
struct chd_context {
  std::unique_ptr<chd::Context> c;
};
struct chd_ciphertext {
  chd::DeviceCt ct;
};
struct chd_evk {
  chd::DeviceEvk k;
};
