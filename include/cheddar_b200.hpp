// cheddar_b200.hpp — header-only C++ mirror of the reference's server-side
// API (scale-snu/cheddar-fhe include/core/Context.h, Container.h) over the C
// ABI of include/cheddar_b200.h.  Method names, argument order and meaning
// follow the reference: results are written into a caller-owned `res`
// (Context.h:101-423).  On failure the reference terminates the process
// (include/common/Assert.h:9-21); this shim throws cheddar_b200::Error
// instead (define CHEDDAR_B200_ABORT_ON_ERROR to print and std::exit like
// the reference).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cheddar_b200.h"

namespace cheddar_b200 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc == CHD_OK) return;
#ifdef CHEDDAR_B200_ABORT_ON_ERROR
  std::fprintf(stderr, "ERROR: %s\n", chd_last_error());
  std::exit(EXIT_FAILURE);
#else
  throw Error(rc, chd_last_error());
#endif
}

class Context;

// Ciphertext<uint32_t> (Container.h:131-175): device residues [np][N] per part.
class Ciphertext {
 public:
  explicit Ciphertext(Context &ctx);
  ~Ciphertext() { chd_ct_destroy(ct_); }
  Ciphertext(const Ciphertext &) = delete;
  Ciphertext &operator=(const Ciphertext &) = delete;
  Ciphertext(Ciphertext &&o) noexcept : ct_(o.ct_) { o.ct_ = nullptr; }

  // Ciphertext::GetNP / HasRx / GetScale / GetNumSlots
  int NumMain() const { return info().num_main; }
  int NumTer() const { return info().num_ter; }
  int NumAux() const { return info().num_aux; }
  bool HasRx() const { return info().has_rx; }
  double GetScale() const { return info().scale; }
  int GetNumSlots() const { return info().num_slots; }

  chd_ciphertext *raw() const { return ct_; }

 private:
  struct Info {
    int num_main, num_ter, num_aux, has_rx;
    double scale;
    int num_slots;
  };
  Info info() const {
    Info i{};
    check(chd_ct_info(ct_, &i.num_main, &i.num_ter, &i.num_aux, &i.has_rx, &i.scale, &i.num_slots));
    return i;
  }
  chd_ciphertext *ct_ = nullptr;
};

// EvaluationKey<uint32_t> (Container.h:283-344): beta pairs over [L + alpha][N].
class EvaluationKey {
 public:
  EvaluationKey(Context &ctx, int beta, const uint32_t *bx, const uint32_t *ax, bool on_device);
  ~EvaluationKey() { chd_evk_destroy(k_); }
  EvaluationKey(const EvaluationKey &) = delete;
  EvaluationKey &operator=(const EvaluationKey &) = delete;
  chd_evk *raw() const { return k_; }

 private:
  chd_evk *k_ = nullptr;
};

// Context<uint32_t> (Context.h:17-424)
class Context {
 public:
  using Ct = Ciphertext;
  using Evk = EvaluationKey;

  // Parameter JSON (unittest/Testbed.h schema) -> Parameter + Context::Create
  static std::shared_ptr<Context> Create(const std::string &param_json, int device = 0) {
    chd_context *c = nullptr;
    check(chd_context_create_json(param_json.c_str(), device, &c));
    return std::shared_ptr<Context>(new Context(c));
  }
  // Parameter(log_degree, base_scale, default_encryption_level, level_config,
  //           main_primes, aux_primes, ter_primes, additional_base)
  static std::shared_ptr<Context> Create(int log_degree, double base_scale, int default_encryption_level,
                                         const std::vector<std::pair<int, int>> &level_config,
                                         const std::vector<uint32_t> &main_primes,
                                         const std::vector<uint32_t> &aux_primes,
                                         const std::vector<uint32_t> &ter_primes = {},
                                         std::pair<int, int> additional_base = {0, 0}, int device = 0) {
    std::vector<int> lc;
    for (auto &p : level_config) {
      lc.push_back(p.first);
      lc.push_back(p.second);
    }
    chd_context *c = nullptr;
    check(chd_context_create(log_degree, base_scale, default_encryption_level, lc.data(),
                             static_cast<int>(level_config.size()), main_primes.data(),
                             static_cast<int>(main_primes.size()), aux_primes.data(),
                             static_cast<int>(aux_primes.size()), ter_primes.empty() ? nullptr : ter_primes.data(),
                             static_cast<int>(ter_primes.size()), additional_base.first, additional_base.second,
                             device, &c));
    return std::shared_ptr<Context>(new Context(c));
  }
  ~Context() { chd_context_destroy(c_); }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;

  chd_context *raw() const { return c_; }
  int MaxLevel() const { return chd_max_level(c_); }
  int Degree() const { return chd_degree(c_); }
  double GetScale(int level) const { return chd_scale(c_, level); }
  double GetRescalePrimeProd(int level) const { return chd_rescale_prime_prod(c_, level); }
  void SetStream(void *cuda_stream) { check(chd_context_set_stream(c_, cuda_stream)); }
  void Synchronize() { check(chd_context_synchronize(c_)); }
  // Base-conversion engine of every ModUp / ModDown (CHD_BCONV_CUDA_CORE,
  // CHD_BCONV_TENSOR_CORE or CHD_BCONV_AUTO); results are bit-identical.
  void SetKeySwitchEngine(int engine) { check(chd_set_ks_engine(c_, engine)); }
  int KeySwitchEngine() const { return chd_get_ks_engine(c_); }
  void SetStreamSplit(bool on) { check(chd_set_stream_split(c_, on ? 1 : 0)); }
  bool StreamSplit() const { return chd_get_stream_split(c_) == 1; }

  // residue import / export ([np][N] per part), host or device pointers
  void Import(Ct &ct, int level, int num_aux, double scale, int num_slots, const uint32_t *bx,
              const uint32_t *ax, const uint32_t *rx = nullptr, bool on_device = false) {
    int m = 0, t = 0;
    check(chd_level_np(c_, level, &m, &t));
    check(chd_ct_import(c_, ct.raw(), m, t, num_aux, rx != nullptr, scale, num_slots, bx, ax, rx, on_device));
  }
  void Export(const Ct &ct, uint32_t *bx, uint32_t *ax, uint32_t *rx = nullptr, bool on_device = false) {
    check(chd_ct_export(c_, ct.raw(), bx, ax, rx, on_device));
  }

  // ---- evaluator (same signatures as the reference) ----
  void Add(Ct &res, const Ct &a, const Ct &b) const { check(chd_add(c_, res.raw(), a.raw(), b.raw())); }
  void Sub(Ct &res, const Ct &a, const Ct &b) const { check(chd_sub(c_, res.raw(), a.raw(), b.raw())); }
  void Neg(Ct &res, const Ct &a) const { check(chd_neg(c_, res.raw(), a.raw())); }
  void Mult(Ct &res, const Ct &a, const Ct &b) const { check(chd_mult(c_, res.raw(), a.raw(), b.raw())); }
  void MultImaginaryUnit(Ct &res, const Ct &a) const { check(chd_mult_imaginary_unit(c_, res.raw(), a.raw())); }
  void Rescale(Ct &res, const Ct &a) const { check(chd_rescale(c_, res.raw(), a.raw())); }
  void Relinearize(Ct &res, const Ct &a, const Evk &key) const {
    check(chd_relinearize(c_, res.raw(), a.raw(), key.raw()));
  }
  void RelinearizeRescale(Ct &res, const Ct &a, const Evk &key) const {
    check(chd_relinearize_rescale(c_, res.raw(), a.raw(), key.raw()));
  }
  void MultKey(Ct &res, const Ct &a, const Evk &key) const { check(chd_mult_key(c_, res.raw(), a.raw(), key.raw())); }
  void HMult(Ct &res, const Ct &a, const Ct &b, const Evk &mult_key, bool rescale = true) const {
    check(chd_hmult(c_, res.raw(), a.raw(), b.raw(), mult_key.raw(), rescale ? 1 : 0));
  }
  void HRot(Ct &res, const Ct &a, const Evk &rot_key, int rot_dist) const {
    check(chd_hrot(c_, res.raw(), a.raw(), rot_key.raw(), rot_dist));
  }
  void HConj(Ct &res, const Ct &a, const Evk &conj_key) const {
    check(chd_hconj(c_, res.raw(), a.raw(), conj_key.raw()));
  }
  void HRotAdd(Ct &res, const Ct &a, const Ct &b, const Evk &rot_key, int rot_dist) const {
    check(chd_hrot_add(c_, res.raw(), a.raw(), b.raw(), rot_key.raw(), rot_dist));
  }
  void Copy(Ct &res, const Ct &a) const { check(chd_copy(c_, res.raw(), a.raw())); }
  // MultUnsafe at a designated level (-1: the lower input level)
  void MultUnsafe(Ct &res, const Ct &a, const Ct &b, int level = -1) const {
    check(chd_mult_unsafe(c_, res.raw(), a.raw(), b.raw(), level));
  }
  // constants: Montgomery residues over const_level's q primes (EncodeConstant)
  void MultUnsafe(Ct &res, const Ct &a, const std::vector<uint32_t> &cx, int const_level, double const_scale,
                  int level = -1) const {
    check(chd_mult_unsafe_const(c_, res.raw(), a.raw(), cx.data(), const_level, const_scale, level));
  }
  void MadUnsafe(Ct &res, const Ct &a, const std::vector<uint32_t> &cx, int const_level, double const_scale) const {
    check(chd_mad_unsafe(c_, res.raw(), a.raw(), cx.data(), const_level, const_scale));
  }
  void Permute(Ct &res, const Ct &a, int rot_dist) const { check(chd_permute(c_, res.raw(), a.raw(), rot_dist)); }
  void PermuteConjugate(Ct &res, const Ct &a) const { check(chd_permute_conjugate(c_, res.raw(), a.raw())); }
  void HConjAdd(Ct &res, const Ct &a, const Ct &b, const Evk &conj_key) const {
    check(chd_hconj_add(c_, res.raw(), a.raw(), b.raw(), conj_key.raw()));
  }
  void LevelDown(Ct &res, const Ct &a, int target_level) const {
    check(chd_level_down(c_, res.raw(), a.raw(), target_level));
  }
  void MultKeyNoModDown(Ct &accum, const Ct &a, const Evk &key) const {
    check(chd_mult_key_no_moddown(c_, accum.raw(), a.raw(), key.raw()));
  }
  // plaintexts: device residues over the ciphertext's primes (chd_encode)
  void Add(Ct &res, const Ct &a, const uint32_t *pt_dev, double pt_scale) const {
    check(chd_add_plain(c_, res.raw(), a.raw(), pt_dev, pt_scale));
  }
  void Sub(Ct &res, const Ct &a, const uint32_t *pt_dev, double pt_scale) const {
    check(chd_sub_plain(c_, res.raw(), a.raw(), pt_dev, pt_scale));
  }
  void Sub(Ct &res, const uint32_t *pt_dev, double pt_scale, const Ct &b) const {
    check(chd_sub_plain_ct(c_, res.raw(), pt_dev, pt_scale, b.raw()));
  }
  void Mult(Ct &res, const Ct &a, const uint32_t *pt_dev, double pt_scale) const {
    check(chd_mult_plain(c_, res.raw(), a.raw(), pt_dev, pt_scale));
  }
  void MultUnsafe(Ct &res, const Ct &a, const uint32_t *pt_dev, int pt_level, int pt_num_aux, double pt_scale,
                  int level = -1) const {
    check(chd_mult_unsafe_plain(c_, res.raw(), a.raw(), pt_dev, pt_level, pt_num_aux, pt_scale, level));
  }
  // constants: Montgomery residues per prime (EncodeConstant)
  void Add(Ct &res, const Ct &a, const std::vector<uint32_t> &cx) const {
    check(chd_add_const(c_, res.raw(), a.raw(), cx.data()));
  }
  void Mult(Ct &res, const Ct &a, const std::vector<uint32_t> &cx, double const_scale) const {
    check(chd_mult_const(c_, res.raw(), a.raw(), cx.data(), const_scale));
  }
  void Sub(Ct &res, const Ct &a, const std::vector<uint32_t> &cx) const {
    check(chd_sub_const(c_, res.raw(), a.raw(), cx.data()));
  }
  void Sub(Ct &res, const std::vector<uint32_t> &cx, double const_scale, const Ct &b) const {
    check(chd_sub_const_ct(c_, res.raw(), cx.data(), const_scale, b.raw()));
  }
  bool IsMultUnsafeCompatible(int level1, int level2) const {
    const int r = chd_mult_unsafe_compatible(c_, level1, level2);
    if (r < 0) throw Error(CHD_ERR_INVALID_ARG, "IsMultUnsafeCompatible: invalid level");
    return r != 0;
  }
  // batched HMult over independent pairs (one fused pipeline per level)
  void HMultBatch(const std::vector<Ct *> &res, const std::vector<const Ct *> &a,
                  const std::vector<const Ct *> &b, const Evk &mult_key, bool rescale = true) const {
    std::vector<chd_ciphertext *> r;
    std::vector<const chd_ciphertext *> x, y;
    for (size_t i = 0; i < res.size(); i++) {
      r.push_back(res[i]->raw());
      x.push_back(a[i]->raw());
      y.push_back(b[i]->raw());
    }
    check(chd_hmult_batch(c_, static_cast<int>(r.size()), r.data(), x.data(), y.data(), mult_key.raw(),
                          rescale ? 1 : 0));
  }

  // ---- encoder (Encoder::Encode / EncodeConstant) ----
  // plaintext [num_q(level) + num_aux][N] at pt_dev (evaluation domain, Montgomery)
  int Encode(uint32_t *pt_dev, int level, double scale, const std::vector<double> &re,
             const std::vector<double> &im, int num_aux = 0) const {
    int slots = 0;
    check(chd_encode(c_, level, scale, re.data(), im.data(), static_cast<int>(re.size()), num_aux, pt_dev, &slots));
    return slots;
  }
  std::vector<uint32_t> EncodeConstant(int level, double scale, double value, int num_aux = 0) const {
    int m = 0, t = 0;
    check(chd_level_np(c_, level, &m, &t));
    std::vector<uint32_t> cx(m + t + num_aux);
    check(chd_encode_const(c_, level, scale, value, num_aux, cx.data()));
    return cx;
  }

  // ---- CUDA graphs of library calls ----
  void BeginGraph() { check(chd_graph_begin(c_)); }
  chd_graph *EndGraph() {
    chd_graph *g = nullptr;
    check(chd_graph_end(c_, &g));
    return g;
  }
  void LaunchGraph(const chd_graph *g) { check(chd_graph_launch(c_, g)); }

 private:
  explicit Context(chd_context *c) : c_(c) {}
  chd_context *c_ = nullptr;
};

// EvkMap (include/core/EvkMap.h): keys by rotation index plus the
// conjugation and multiplication keys (borrowed; they must outlive the map)
class EvkMap {
 public:
  explicit EvkMap(Context &ctx) { check(chd_evk_map_create(ctx.raw(), &m_)); }
  ~EvkMap() { chd_evk_map_destroy(m_); }
  EvkMap(const EvkMap &) = delete;
  EvkMap &operator=(const EvkMap &) = delete;
  void AddRotationKey(int rot_idx, const EvaluationKey &k) { check(chd_evk_map_set_rotation(m_, rot_idx, k.raw())); }
  void SetConjugationKey(const EvaluationKey &k) { check(chd_evk_map_set_conjugation(m_, k.raw())); }
  void SetMultiplicationKey(const EvaluationKey &k) { check(chd_evk_map_set_mult(m_, k.raw())); }
  void SetDenseToSparseKey(const EvaluationKey &k) { check(chd_evk_map_set_dense_to_sparse(m_, k.raw())); }
  void SetSparseToDenseKey(const EvaluationKey &k) { check(chd_evk_map_set_sparse_to_dense(m_, k.raw())); }
  chd_evk_map *raw() const { return m_; }

 private:
  chd_evk_map *m_ = nullptr;
};

// BootContext (include/extension/BootContext.h) for one slot count:
// PrepareEvalMod + PrepareEvalSpecialFFT at construction, then Boot.
class BootContext {
 public:
  // PrepareEvalSpecialFFT(num_slots, variant): variant CHD_BOOT_NORMAL,
  // CHD_BOOT_IMAGINARY_REMOVING or CHD_BOOT_MERGE_TWO_REAL
  BootContext(Context &ctx, int num_slots, int num_cts_levels = 4, int num_stc_levels = 3,
              int log_message_ratio = 5, int variant = CHD_BOOT_NORMAL)
      : ctx_(ctx) {
    check(chd_boot_create_variant(ctx.raw(), num_slots, variant, num_cts_levels, num_stc_levels, log_message_ratio,
                                  &b_));
  }
  ~BootContext() { chd_boot_destroy(b_); }
  BootContext(const BootContext &) = delete;
  BootContext &operator=(const BootContext &) = delete;
  // AddRequiredRotations: the rotation keys the client must provide
  std::vector<int> RequiredRotations(bool min_ks = false) const {
    int n = 0;
    check(chd_boot_rotations(b_, min_ks ? 1 : 0, nullptr, 0, &n));
    std::vector<int> r(n);
    check(chd_boot_rotations(b_, min_ks ? 1 : 0, r.data(), n, &n));
    return r;
  }
  int GetEndLevel() const {
    int lv[5];
    check(chd_boot_levels(b_, lv, nullptr));
    return lv[3];
  }
  void ModUpToMax(Ciphertext &res, const Ciphertext &in, const EvkMap &evk_map) const {
    check(chd_modup_to_max(ctx_.raw(), res.raw(), in.raw(), evk_map.raw()));
  }
  void Boot(Ciphertext &res, const Ciphertext &in, const EvkMap &evk_map, bool min_ks = false) {
    check(chd_boot_run(ctx_.raw(), b_, res.raw(), in.raw(), evk_map.raw(), min_ks ? 1 : 0));
  }
  // every ciphertext of the batch in one call (key switches batched)
  void BootBatch(const std::vector<Ciphertext *> &res, const std::vector<const Ciphertext *> &in,
                 const EvkMap &evk_map, bool min_ks = false) {
    std::vector<chd_ciphertext *> r;
    std::vector<const chd_ciphertext *> x;
    for (size_t i = 0; i < res.size(); i++) {
      r.push_back(res[i]->raw());
      x.push_back(in[i]->raw());
    }
    check(chd_boot_run_batch(ctx_.raw(), b_, static_cast<int>(r.size()), r.data(), x.data(), evk_map.raw(),
                             min_ks ? 1 : 0));
  }

 private:
  Context &ctx_;
  chd_boot *b_ = nullptr;
};

inline Ciphertext::Ciphertext(Context &ctx) { check(chd_ct_create(ctx.raw(), &ct_)); }

// ---- the 64-bit word path: Context<uint64_t> (Context.cpp:952) ----

class Context64;

// Ciphertext<uint64_t>: uint64 residues [np][N] per part (rx after Mult)
class Ciphertext64 {
 public:
  explicit Ciphertext64(Context64 &ctx);
  ~Ciphertext64() { chd64_ct_destroy(ct_); }
  Ciphertext64(const Ciphertext64 &) = delete;
  Ciphertext64 &operator=(const Ciphertext64 &) = delete;
  Ciphertext64(Ciphertext64 &&o) noexcept : ct_(o.ct_) { o.ct_ = nullptr; }
  int NumMain() const { return info().num_main; }
  int NumTer() const { return info().num_ter; }
  bool HasRx() const { return chd64_ct_has_rx(ct_) == 1; }
  double GetScale() const { return info().scale; }
  int GetNumSlots() const { return info().num_slots; }
  chd64_ciphertext *raw() const { return ct_; }

 private:
  struct Info {
    int num_main, num_ter;
    double scale;
    int num_slots;
  };
  Info info() const {
    Info i{};
    check(chd64_ct_info(ct_, &i.num_main, &i.num_ter, &i.scale, &i.num_slots));
    return i;
  }
  chd64_ciphertext *ct_ = nullptr;
};

// EvaluationKey<uint64_t>: beta pairs over [L + alpha][N]
class EvaluationKey64 {
 public:
  EvaluationKey64(Context64 &ctx, int beta, const uint64_t *bx, const uint64_t *ax, bool on_device);
  ~EvaluationKey64() { chd64_evk_destroy(k_); }
  EvaluationKey64(const EvaluationKey64 &) = delete;
  EvaluationKey64 &operator=(const EvaluationKey64 &) = delete;
  chd64_evk *raw() const { return k_; }

 private:
  chd64_evk *k_ = nullptr;
};

// Context<uint64_t> (Context.h:17-424 with word = uint64_t)
class Context64 {
 public:
  using Ct = Ciphertext64;
  using Evk = EvaluationKey64;
  static std::shared_ptr<Context64> Create(const std::string &param_json, int device = 0) {
    chd64_context *c = nullptr;
    check(chd64_context_create_json(param_json.c_str(), device, &c));
    return std::shared_ptr<Context64>(new Context64(c));
  }
  ~Context64() { chd64_context_destroy(c_); }
  Context64(const Context64 &) = delete;
  Context64 &operator=(const Context64 &) = delete;

  chd64_context *raw() const { return c_; }
  int MaxLevel() const { return chd64_max_level(c_); }
  double GetScale(int level) const { return chd64_scale(c_, level); }
  void SetStream(void *cuda_stream) { check(chd64_context_set_stream(c_, cuda_stream)); }
  void Synchronize() { check(chd64_context_synchronize(c_)); }

  void Import(Ct &ct, int level, double scale, int num_slots, const uint64_t *bx, const uint64_t *ax,
              const uint64_t *rx = nullptr, bool on_device = false) {
    check(chd64_ct_import(c_, ct.raw(), level, scale, num_slots, bx, ax, on_device ? 1 : 0));
    if (rx) check(chd64_ct_set_rx(c_, ct.raw(), rx, on_device ? 1 : 0));
  }
  void Export(const Ct &ct, uint64_t *bx, uint64_t *ax, uint64_t *rx = nullptr) {
    check(chd64_ct_export(c_, ct.raw(), bx, ax));
    if (rx && ct.HasRx()) check(chd64_ct_export_rx(c_, ct.raw(), rx));
  }
  // Encoder<uint64_t>::EncodeConstant: one Montgomery word per prime
  std::vector<uint64_t> EncodeConstant(int level, double scale, double value, int num_aux = 0) {
    int m = 0, t = 0;
    check(chd64_level_np(c_, level, &m, &t));
    std::vector<uint64_t> cx(m + t + num_aux);
    check(chd64_encode_const(c_, level, scale, value, num_aux, cx.data()));
    return cx;
  }

  // ---- evaluator (same signatures as the reference; constants as words) ----
  void Copy(Ct &res, const Ct &a) const { check(chd64_copy(c_, res.raw(), a.raw())); }
  void Add(Ct &res, const Ct &a, const Ct &b) const { check(chd64_add(c_, res.raw(), a.raw(), b.raw())); }
  void Sub(Ct &res, const Ct &a, const Ct &b) const { check(chd64_sub(c_, res.raw(), a.raw(), b.raw())); }
  void Neg(Ct &res, const Ct &a) const { check(chd64_neg(c_, res.raw(), a.raw())); }
  void Mult(Ct &res, const Ct &a, const Ct &b) const { check(chd64_mult(c_, res.raw(), a.raw(), b.raw())); }
  void Mult(Ct &res, const Ct &a, const std::vector<uint64_t> &cx, double const_scale) const {
    check(chd64_mult_const(c_, res.raw(), a.raw(), cx.data(), const_scale));
  }
  void Add(Ct &res, const Ct &a, const std::vector<uint64_t> &cx) const {
    check(chd64_add_const(c_, res.raw(), a.raw(), cx.data()));
  }
  void MultImaginaryUnit(Ct &res, const Ct &a) const { check(chd64_mult_imaginary_unit(c_, res.raw(), a.raw())); }
  void Rescale(Ct &res, const Ct &a) const { check(chd64_rescale(c_, res.raw(), a.raw())); }
  void Relinearize(Ct &res, const Ct &a, const Evk &key) const {
    check(chd64_relinearize(c_, res.raw(), a.raw(), key.raw(), 0));
  }
  void RelinearizeRescale(Ct &res, const Ct &a, const Evk &key) const {
    check(chd64_relinearize(c_, res.raw(), a.raw(), key.raw(), 1));
  }
  void MultKey(Ct &res, const Ct &a, const Evk &key) const { check(chd64_mult_key(c_, res.raw(), a.raw(), key.raw())); }
  void Permute(Ct &res, const Ct &a, int rot_dist) const { check(chd64_permute(c_, res.raw(), a.raw(), rot_dist, 0)); }
  void PermuteConjugate(Ct &res, const Ct &a) const { check(chd64_permute(c_, res.raw(), a.raw(), 0, 1)); }
  void HMult(Ct &res, const Ct &a, const Ct &b, const Evk &mult_key, bool rescale = true) const {
    check(chd64_hmult(c_, res.raw(), a.raw(), b.raw(), mult_key.raw(), rescale ? 1 : 0));
  }
  void HRot(Ct &res, const Ct &a, const Evk &rot_key, int rot_dist) const {
    check(chd64_hrot(c_, res.raw(), a.raw(), rot_key.raw(), rot_dist));
  }
  void HConj(Ct &res, const Ct &a, const Evk &conj_key) const {
    check(chd64_hconj(c_, res.raw(), a.raw(), conj_key.raw()));
  }
  void HRotAdd(Ct &res, const Ct &a, const Ct &b, const Evk &rot_key, int rot_dist) const {
    check(chd64_hrot_add(c_, res.raw(), a.raw(), b.raw(), rot_key.raw(), rot_dist));
  }
  void HConjAdd(Ct &res, const Ct &a, const Ct &b, const Evk &conj_key) const {
    check(chd64_hconj_add(c_, res.raw(), a.raw(), b.raw(), conj_key.raw()));
  }
  void LevelDown(Ct &res, const Ct &a, int target_level) const {
    check(chd64_level_down(c_, res.raw(), a.raw(), target_level));
  }

 private:
  explicit Context64(chd64_context *c) : c_(c) {}
  chd64_context *c_ = nullptr;
};

inline Ciphertext64::Ciphertext64(Context64 &ctx) { check(chd64_ct_create(ctx.raw(), &ct_)); }

inline EvaluationKey64::EvaluationKey64(Context64 &ctx, int beta, const uint64_t *bx, const uint64_t *ax,
                                        bool on_device) {
  check(chd64_evk_create(ctx.raw(), beta, bx, ax, on_device ? 1 : 0, &k_));
}

inline EvaluationKey::EvaluationKey(Context &ctx, int beta, const uint32_t *bx, const uint32_t *ax,
                                    bool on_device) {
  check(chd_evk_create(ctx.raw(), beta, bx, ax, on_device ? 1 : 0, &k_));
}

}  // namespace cheddar_b200
