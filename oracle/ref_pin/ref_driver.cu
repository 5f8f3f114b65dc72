// Reference driver: a C ABI over the reference's own C++/CUDA library
// (src/core, src/extension, src/UserInterface.cu compiled for sm_100a from
// the reference tree by oracle/Makefile target `reflib`), so that Python tests
// and the bench can run the reference's evaluator on the same residues and
// keys as this library and the oracle.  Test infrastructure only: nothing in
// the product links it.
//
// What it exposes, each a thin call into the reference:
//  * context creation from the parameter-JSON fields (unittest/Testbed.h:94-226
//    parses the same fields), with BootContext when `boot` is set;
//  * the reference's test client (UserInterface.cu: secrets, mult / conj /
//    sparse-secret keys at construction, rotation keys on request), with
//    every key generated over the full key basis (UserInterface.cu:523-541
//    at the maximum level) and exported as beta pairs [beta][np][N];
//  * ciphertext import/export through the public bx_/ax_/rx_ members
//    (include/core/Container.h:154-156), encryption and decryption+decoding;
//  * HMult, HRot, HConj, Relinearize, Rescale (Context.cpp), raw NTT / INTT
//    (NTT.cu:606-741), ModUp / ModDown / Rescale / ModDownAndRescale
//    (ModSwitch.cu:429-684), hoisted baby steps (Hoist.cu:578-691) and Boot
//    (BootContext.cpp:299-365);
//  * device timing of HMult, HRot, the NTT round trip and Boot with CUDA
//    events on the legacy stream the reference issues its work on;
//  * the 64-bit word path (refx64_*): Context<uint64_t> from the same JSON
//    fields, raw NTT / ModUp / ModDown, and HMult / HRot on imported
//    ciphertexts and keys (host [np][N] uint64 buffers).
//
// The reference reports failures by exiting the process
// (include/common/Assert.h:9-21); callers must pass valid inputs.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "UserInterface.h"
#include "common/CommonUtils.h"
#include "core/EvkRequest.h"
#include "extension/BootContext.h"
#include "extension/Hoist.h"

using namespace cheddar;
using word = uint32_t;

namespace {

struct RefCtx {
  std::unique_ptr<Parameter<word>> param;
  ContextPtr<word> ctx;
  std::shared_ptr<BootContext<word>> boot;
  std::unique_ptr<UserInterface<word>> ui;
  bool evalmod_prepared = false;
  std::set<int> fft_prepared;
  int degree = 0;
};

double test_scale(const RefCtx &R, int level) {
  // unittest/Testbed.h:231-238 (DetermineScale)
  if (level <= R.param->default_encryption_level_) return R.param->GetScale(level);
  return R.param->GetRescalePrimeProd(level);
}

size_t poly_words(const NPInfo &np, int degree) {
  return static_cast<size_t>(np.GetNumTotal()) * degree;
}

void copy_in(DeviceVector<word> &dst, const uint32_t *src, size_t words) {
  dst.resize(static_cast<int>(words));
  cudaMemcpy(dst.data(), src, words * sizeof(word), cudaMemcpyHostToDevice);
}

void copy_out(uint32_t *dst, const DeviceVector<word> &src, size_t words) {
  cudaMemcpy(dst, src.data(), words * sizeof(word), cudaMemcpyDeviceToHost);
}

const EvaluationKey<word> *find_key(const RefCtx &R, int key_idx) {
  const EvkMap<word> &m = R.ui->GetEvkMap();
  auto it = m.find(key_idx);
  return it == m.end() ? nullptr : &it->second;
}

int last_cuda() {
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : -static_cast<int>(e);
}

template <typename F>
int time_loop(int warmup, int iters, F &&f, float *ms) {
  for (int i = 0; i < warmup; i++) f();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0, cudaStreamLegacy);
  for (int i = 0; i < iters; i++) f();
  cudaEventRecord(e1, cudaStreamLegacy);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return last_cuda();
}

}  // namespace

extern "C" {

// Special key indices of include/core/EvkMap.h:16-19.
int refx_key_index_mult() { return EvkMap<word>::kMultiplicationKeyIndex; }
int refx_key_index_conj() { return EvkMap<word>::kConjugationKeyIndex; }
int refx_key_index_dts() { return EvkMap<word>::kDenseToSparseKeyIndex; }
int refx_key_index_std() { return EvkMap<word>::kSparseToDenseKeyIndex; }

int refx_create(int log_degree, int log_scale, int enc_level, int n_levels, const int *level_pairs,
                const uint32_t *main_primes, int n_main, const uint32_t *aux_primes, int n_aux,
                const uint32_t *ter_primes, int n_ter, int add_main, int add_ter, int dense_h,
                int sparse_h, int boot, int num_cts, int num_stc, void **out) {
  auto *R = new RefCtx();
  std::vector<std::pair<int, int>> cfg;
  for (int i = 0; i < n_levels; i++) cfg.emplace_back(level_pairs[2 * i], level_pairs[2 * i + 1]);
  std::vector<word> m(main_primes, main_primes + n_main), a(aux_primes, aux_primes + n_aux),
      t(ter_primes, ter_primes + n_ter);
  double scale = static_cast<double>(UINT64_C(1) << log_scale);
  R->param = std::make_unique<Parameter<word>>(log_degree, scale, enc_level, cfg, m, a, t,
                                               std::make_pair(add_main, add_ter));
  if (dense_h > 0) R->param->SetDenseHammingWeight(dense_h);
  if (sparse_h > 0) R->param->SetSparseHammingWeight(sparse_h);
  if (boot) {
    R->boot = BootContext<word>::Create(*R->param,
                                        BootParameter(R->param->max_level_, num_cts, num_stc));
    R->ctx = R->boot;
  } else {
    R->ctx = Context<word>::Create(*R->param);
  }
  R->ui = std::make_unique<UserInterface<word>>(R->ctx);
  R->degree = R->param->degree_;
  *out = R;
  return last_cuda();
}

void refx_destroy(void *p) {
  auto *R = static_cast<RefCtx *>(p);
  cudaDeviceSynchronize();
  R->ui.reset();
  R->boot.reset();
  R->ctx.reset();
  R->param.reset();
  delete R;
}

int refx_max_level(void *p) { return static_cast<RefCtx *>(p)->param->max_level_; }
int refx_alpha(void *p) { return static_cast<RefCtx *>(p)->param->alpha_; }
int refx_dnum(void *p) { return static_cast<RefCtx *>(p)->param->dnum_; }

void refx_level_np(void *p, int level, int num_aux, int *num_main, int *num_ter) {
  NPInfo np = static_cast<RefCtx *>(p)->param->LevelToNP(level, num_aux);
  *num_main = np.num_main_;
  *num_ter = np.num_ter_;
}

double refx_test_scale(void *p, int level) { return test_scale(*static_cast<RefCtx *>(p), level); }
double refx_scale(void *p, int level) { return static_cast<RefCtx *>(p)->param->GetScale(level); }

// Prime vector of an NP (Parameter.cu GetPrimeVector): the row order of a
// polynomial over that NP.
int refx_prime_vector(void *p, int num_main, int num_ter, int num_aux, uint32_t *out) {
  auto v = static_cast<RefCtx *>(p)->param->GetPrimeVector(NPInfo(num_main, num_ter, num_aux));
  for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
  return static_cast<int>(v.size());
}

// ---- keys ----

// Rotation key over the full key basis (UserInterface.cu:278-305, max_level
// = the parameter's maximum level).
int refx_prepare_rotation(void *p, int rot_idx) {
  auto *R = static_cast<RefCtx *>(p);
  R->ui->PrepareRotationKey(rot_idx, R->param->max_level_);
  return last_cuda();
}

int refx_key_shape(void *p, int key_idx, int *beta, int *num_main, int *num_ter, int *num_aux) {
  const EvaluationKey<word> *k = find_key(*static_cast<RefCtx *>(p), key_idx);
  if (k == nullptr) return -1;
  NPInfo np = k->GetNP();
  *beta = k->GetBeta();
  *num_main = np.num_main_;
  *num_ter = np.num_ter_;
  *num_aux = np.num_aux_;
  return 0;
}

// bx, ax: host [beta][np.total][N].
int refx_key_export(void *p, int key_idx, uint32_t *bx, uint32_t *ax) {
  auto *R = static_cast<RefCtx *>(p);
  const EvaluationKey<word> *k = find_key(*R, key_idx);
  if (k == nullptr) return -1;
  size_t w = poly_words(k->GetNP(), R->degree);
  for (int i = 0; i < k->GetBeta(); i++) {
    copy_out(bx + i * w, k->bx_.at(i), w);
    copy_out(ax + i * w, k->ax_.at(i), w);
  }
  return last_cuda();
}

// ---- ciphertexts ----

void *refx_ct_new() { return new Ciphertext<word>(); }
void refx_ct_free(void *c) {
  cudaDeviceSynchronize();
  delete static_cast<Ciphertext<word> *>(c);
}

void refx_ct_info(void *c, int *num_main, int *num_ter, int *num_aux, int *has_rx, double *scale,
                  int *num_slots) {
  auto *ct = static_cast<Ciphertext<word> *>(c);
  NPInfo np = ct->GetNP();
  *num_main = np.num_main_;
  *num_ter = np.num_ter_;
  *num_aux = np.num_aux_;
  *has_rx = ct->HasRx() ? 1 : 0;
  *scale = ct->GetScale();
  *num_slots = ct->GetNumSlots();
}

int refx_ct_export(void *p, void *c, uint32_t *bx, uint32_t *ax, uint32_t *rx) {
  auto *R = static_cast<RefCtx *>(p);
  auto *ct = static_cast<Ciphertext<word> *>(c);
  size_t w = poly_words(ct->GetNP(), R->degree);
  copy_out(bx, ct->bx_, w);
  copy_out(ax, ct->ax_, w);
  if (ct->HasRx() && rx != nullptr) copy_out(rx, ct->rx_, w);
  return last_cuda();
}

int refx_ct_import(void *p, void *c, int num_main, int num_ter, int num_aux, double scale, int num_slots,
                   const uint32_t *bx, const uint32_t *ax) {
  auto *R = static_cast<RefCtx *>(p);
  auto *ct = static_cast<Ciphertext<word> *>(c);
  NPInfo np(num_main, num_ter, num_aux);
  ct->RemoveRx();
  ct->ModifyNP(np);
  ct->SetScale(scale);
  ct->SetNumSlots(num_slots);
  size_t w = poly_words(np, R->degree);
  copy_in(ct->bx_, bx, w);
  copy_in(ct->ax_, ax, w);
  return last_cuda();
}

// Encode (scale of unittest/Testbed.h:231-238) and encrypt a message of
// num_slots complex slots at `level`.
int refx_ct_encrypt(void *p, void *c, int level, const double *re, const double *im, int num_slots) {
  auto *R = static_cast<RefCtx *>(p);
  std::vector<Complex> msg(num_slots);
  for (int i = 0; i < num_slots; i++) msg[i] = Complex(re[i], im[i]);
  Plaintext<word> pt;
  R->ctx->encoder_.Encode(pt, level, test_scale(*R, level), msg);
  R->ui->Encrypt(*static_cast<Ciphertext<word> *>(c), pt);
  return last_cuda();
}

int refx_decrypt_decode(void *p, void *c, double *re, double *im) {
  auto *R = static_cast<RefCtx *>(p);
  auto *ct = static_cast<Ciphertext<word> *>(c);
  Plaintext<word> pt;
  R->ui->Decrypt(pt, *ct);
  std::vector<Complex> msg;
  R->ctx->encoder_.Decode(msg, pt);
  for (size_t i = 0; i < msg.size(); i++) {
    re[i] = msg[i].real();
    im[i] = msg[i].imag();
  }
  return last_cuda();
}

// UserInterface::Decrypt (UserInterface.cu:185-206): plaintext residues
// [np.total][N] (evaluation domain, Montgomery form) of a ciphertext.
int refx_decrypt(void *p, void *c, uint32_t *pt_out, double *scale, int *num_slots) {
  auto *R = static_cast<RefCtx *>(p);
  Plaintext<word> pt;
  R->ui->Decrypt(pt, *static_cast<Ciphertext<word> *>(c));
  copy_out(pt_out, pt.mx_, poly_words(pt.GetNP(), R->degree));
  *scale = pt.GetScale();
  *num_slots = pt.GetNumSlots();
  return last_cuda();
}

// Encoder::Decode (Encode.cpp:45-70, 192-248) of plaintext residues at a
// level (no aux primes), scale and slot count.
int refx_decode(void *p, int level, double scale, int num_slots, const uint32_t *pt_host, double *re,
                double *im) {
  auto *R = static_cast<RefCtx *>(p);
  Plaintext<word> pt;
  NPInfo np = R->param->LevelToNP(level);
  pt.ModifyNP(np);
  pt.SetScale(scale);
  pt.SetNumSlots(num_slots);
  copy_in(pt.mx_, pt_host, poly_words(np, R->degree));
  std::vector<Complex> msg;
  R->ctx->encoder_.Decode(msg, pt);
  for (size_t i = 0; i < msg.size(); i++) {
    re[i] = msg[i].real();
    im[i] = msg[i].imag();
  }
  return last_cuda();
}

// Encoded plaintext residues (Encode.cpp:135-190) of a message at a level,
// scale and number of aux primes: out = [np.total][N].
int refx_encode(void *p, int level, double scale, const double *re, const double *im, int num_slots,
                int num_aux, uint32_t *out) {
  auto *R = static_cast<RefCtx *>(p);
  std::vector<Complex> msg(num_slots);
  for (int i = 0; i < num_slots; i++) msg[i] = Complex(re[i], im[i]);
  Plaintext<word> pt;
  R->ctx->encoder_.Encode(pt, level, scale, msg, num_aux);
  copy_out(out, pt.mx_, poly_words(pt.GetNP(), R->degree));
  return last_cuda();
}

// ---- evaluator ----

int refx_hmult(void *p, void *res, void *a, void *b, int rescale) {
  auto *R = static_cast<RefCtx *>(p);
  R->ctx->HMult(*static_cast<Ciphertext<word> *>(res), *static_cast<Ciphertext<word> *>(a),
                *static_cast<Ciphertext<word> *>(b), R->ui->GetMultiplicationKey(), rescale != 0);
  return last_cuda();
}

int refx_hrot(void *p, void *res, void *a, int rot) {
  auto *R = static_cast<RefCtx *>(p);
  int idx = rot < 0 ? R->degree / 2 + rot : rot;
  R->ctx->HRot(*static_cast<Ciphertext<word> *>(res), *static_cast<Ciphertext<word> *>(a),
               R->ui->GetRotationKey(idx), rot);
  return last_cuda();
}

int refx_hconj(void *p, void *res, void *a) {
  auto *R = static_cast<RefCtx *>(p);
  R->ctx->HConj(*static_cast<Ciphertext<word> *>(res), *static_cast<Ciphertext<word> *>(a),
                R->ui->GetConjugationKey());
  return last_cuda();
}

int refx_rescale(void *p, void *res, void *a) {
  auto *R = static_cast<RefCtx *>(p);
  R->ctx->Rescale(*static_cast<Ciphertext<word> *>(res), *static_cast<Ciphertext<word> *>(a));
  return last_cuda();
}

// Other Context operations by name (Context.h:101-423): one input,
// res = op(a[, arg]).
int refx_unary(void *p, const char *op, void *res, void *a, int arg) {
  auto *R = static_cast<RefCtx *>(p);
  auto &Res = *static_cast<Ciphertext<word> *>(res);
  auto &A = *static_cast<Ciphertext<word> *>(a);
  const std::string o(op);
  if (o == "Neg")
    R->ctx->Neg(Res, A);
  else if (o == "MultImaginaryUnit")
    R->ctx->MultImaginaryUnit(Res, A);
  else if (o == "LevelDown")
    R->ctx->LevelDown(Res, A, arg);
  else if (o == "Relinearize")
    R->ctx->Relinearize(Res, A, R->ui->GetMultiplicationKey());
  else if (o == "RelinearizeRescale")
    R->ctx->RelinearizeRescale(Res, A, R->ui->GetMultiplicationKey());
  else if (o == "MultKeyRot")
    R->ctx->MultKey(Res, A, R->ui->GetRotationKey(arg));
  else if (o == "Permute")
    R->ctx->Permute(Res, A, arg);
  else if (o == "PermuteConjugate")
    R->ctx->PermuteConjugate(Res, A);
  else if (o == "Copy")
    R->ctx->Copy(Res, A);
  else
    return -2;
  return last_cuda();
}

// Two inputs: res = op(a, b[, arg]).
int refx_binary(void *p, const char *op, void *res, void *a, void *b, int arg) {
  auto *R = static_cast<RefCtx *>(p);
  auto &Res = *static_cast<Ciphertext<word> *>(res);
  auto &A = *static_cast<Ciphertext<word> *>(a);
  auto &B = *static_cast<Ciphertext<word> *>(b);
  const std::string o(op);
  if (o == "Add")
    R->ctx->Add(Res, A, B);
  else if (o == "Sub")
    R->ctx->Sub(Res, A, B);
  else if (o == "Mult")
    R->ctx->Mult(Res, A, B);
  else if (o == "MultUnsafe")
    R->ctx->MultUnsafe(Res, A, B, arg);
  else if (o == "HRotAdd")
    R->ctx->HRotAdd(Res, A, B, R->ui->GetRotationKey(arg), arg);
  else if (o == "HConjAdd")
    R->ctx->HConjAdd(Res, A, B, R->ui->GetConjugationKey());
  else
    return -2;
  return last_cuda();
}

// ---- raw NTT / ModSwitch on [np][N] host buffers ----

// NTT (inverse = 0) or INTT (inverse = 1) of `count` polynomials over
// NP(num_main, num_ter, num_aux), in place on the host buffer.
int refx_ntt(void *p, int num_main, int num_ter, int num_aux, uint32_t *data, int count, int inverse,
             int montgomery) {
  auto *R = static_cast<RefCtx *>(p);
  NPInfo np(num_main, num_ter, num_aux);
  size_t w = poly_words(np, R->degree);
  DeviceVector<word> src(static_cast<int>(w)), dst(static_cast<int>(w));
  for (int k = 0; k < count; k++) {
    cudaMemcpy(src.data(), data + k * w, w * 4, cudaMemcpyHostToDevice);
    DvView<word> dv = dst.View(num_aux * R->degree);
    DvConstView<word> sv = src.ConstView(num_aux * R->degree);
    if (inverse)
      R->ctx->ntt_handler_.INTT(dv, np, sv, montgomery != 0);
    else
      R->ctx->ntt_handler_.NTT(dv, np, sv, montgomery != 0);
    cudaMemcpy(data + k * w, dst.data(), w * 4, cudaMemcpyDeviceToHost);
  }
  return last_cuda();
}

// ModUp of a level-`level` polynomial (q primes, evaluation domain):
// out = beta polynomials over q + alpha primes, [beta][q + alpha][N].
int refx_modup(void *p, int level, const uint32_t *src, uint32_t *out) {
  auto *R = static_cast<RefCtx *>(p);
  NPInfo np = R->param->LevelToNP(level);
  int alpha = R->param->alpha_;
  int q = np.GetNumQ();
  int offset = R->param->GetMaxNumTer() - np.num_ter_;
  int beta = DivCeil(q + offset, alpha);
  size_t nq = static_cast<size_t>(q) * R->degree, nqp = static_cast<size_t>(q + alpha) * R->degree;
  DeviceVector<word> s(static_cast<int>(nq));
  cudaMemcpy(s.data(), src, nq * 4, cudaMemcpyHostToDevice);
  std::vector<DeviceVector<word>> tmp;
  std::vector<DvView<word>> views;
  for (int i = 0; i < beta; i++) tmp.emplace_back(static_cast<int>(nqp));
  for (int i = 0; i < beta; i++) views.push_back(tmp[i].View(alpha * R->degree));
  R->ctx->mod_switch_handlers_.at(level).ModUp(views, s.ConstView());
  for (int i = 0; i < beta; i++) copy_out(out + i * nqp, tmp[i], nqp);
  return last_cuda();
}

// kind 0 = ModDown (q+alpha -> q), 1 = Rescale (q -> q of level-1),
// 2 = ModDownAndRescale (q+alpha -> q of level-1).  src over the source NP,
// out over the destination NP.
int refx_moddown(void *p, int level, int kind, const uint32_t *src, uint32_t *out) {
  auto *R = static_cast<RefCtx *>(p);
  int alpha = R->param->alpha_;
  NPInfo np = R->param->LevelToNP(level);
  NPInfo src_np = np;
  if (kind != 1) src_np.num_aux_ = alpha;
  NPInfo dst_np = kind == 0 ? np : R->param->LevelToNP(level - 1);
  size_t ws = poly_words(src_np, R->degree), wd = poly_words(dst_np, R->degree);
  DeviceVector<word> s(static_cast<int>(ws)), d(static_cast<int>(wd));
  cudaMemcpy(s.data(), src, ws * 4, cudaMemcpyHostToDevice);
  DvView<word> dv = d.View();
  DvConstView<word> sv = s.ConstView(src_np.num_aux_ * R->degree);
  const auto &ms = R->ctx->mod_switch_handlers_.at(level);
  if (kind == 0)
    ms.ModDown(dv, sv);
  else if (kind == 1)
    ms.Rescale(dv, sv);
  else
    ms.ModDownAndRescale(dv, sv);
  copy_out(out, d, wd);
  return last_cuda();
}

// ---- hoisted baby steps (Hoist.cu:578-691) ----

// Rotations `rots` (each in [1, N/2), distinct, keys prepared) of one
// ciphertext at its level, left in basis Q u P: outs[i] receives rotation
// rots[i].  The plaintexts a hoisting map needs are zero here: only the baby
// steps are evaluated.
int refx_hoisted_baby_steps(void *p, void *in, const int *rots, int n, void **outs) {
  auto *R = static_cast<RefCtx *>(p);
  auto *ct = static_cast<Ciphertext<word> *>(in);
  int level = R->param->NPToLevel(ct->GetNP());
  PlainHoistMap map;
  Message zero(ct->GetNumSlots(), Complex(0, 0));
  for (int i = 0; i < n; i++) map[0][rots[i]] = zero;
  HoistHandler<word> h(R->ctx, map, level, ct->GetScale(), true);
  std::map<int, Ciphertext<word>> bs;
  h.EvaluateBabyStep(R->ctx, bs, *ct, R->ui->GetEvkMap(), false);
  for (int i = 0; i < n; i++) {
    *static_cast<Ciphertext<word> *>(outs[i]) = std::move(bs.at(rots[i]));
  }
  return last_cuda();
}

// ---- bootstrapping ----

// PrepareEvalMod (once), PrepareEvalSpecialFFT(num_slots) and the rotation
// keys of AddRequiredRotations for hoisted and min-KS evaluation
// (unittest/Bootstrapping.cpp:10-17), every key over the full basis.
// rots_out (capacity cap) receives the distinct rotation indices.
int refx_boot_prepare(void *p, int num_slots, int *rots_out, int cap, int *n_rots) {
  auto *R = static_cast<RefCtx *>(p);
  if (!R->boot) return -1;
  if (!R->evalmod_prepared) {
    R->boot->PrepareEvalMod();
    R->evalmod_prepared = true;
  }
  if (!R->fft_prepared.count(num_slots)) {
    R->boot->PrepareEvalSpecialFFT(num_slots);
    R->fft_prepared.insert(num_slots);
  }
  EvkRequest req;
  R->boot->AddRequiredRotations(req, num_slots, false);
  R->boot->AddRequiredRotations(req, num_slots, true);
  std::set<int> rots;
  for (const auto &kv : req) {
    if (kv.first == 0) continue;
    rots.insert(kv.first < 0 ? -kv.first : kv.first);
  }
  int k = 0;
  for (int r : rots) {
    R->ui->PrepareRotationKey(r, R->param->max_level_);
    if (k < cap) rots_out[k] = r;
    k++;
  }
  *n_rots = k;
  return last_cuda();
}

int refx_boot(void *p, void *res, void *in, int min_ks) {
  auto *R = static_cast<RefCtx *>(p);
  if (!R->boot) return -1;
  R->boot->Boot(*static_cast<Ciphertext<word> *>(res), *static_cast<Ciphertext<word> *>(in),
                R->ui->GetEvkMap(), min_ks != 0);
  return last_cuda();
}

// ---- device timing (CUDA events on the legacy stream) ----


// Total device time of `iters` HMult+relin(+rescale) calls, res != inputs.
int refx_time_hmult(void *p, void *a, void *b, int rescale, int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx *>(p);
  Ciphertext<word> res;
  const auto &key = R->ui->GetMultiplicationKey();
  auto &A = *static_cast<Ciphertext<word> *>(a);
  auto &B = *static_cast<Ciphertext<word> *>(b);
  return time_loop(warmup, iters, [&] { R->ctx->HMult(res, A, B, key, rescale != 0); }, ms);
}

// Total device time of `iters` passes over n distinct (a[i], b[i]) pairs,
// one HMult each (res != inputs): n pairs whose inputs exceed L2 keep the
// timing free of cache reuse between calls.
int refx_time_hmult_set(void *p, void **a, void **b, int n, int rescale, int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx *>(p);
  std::vector<Ciphertext<word>> res(n);
  const auto &key = R->ui->GetMultiplicationKey();
  return time_loop(
      warmup, iters,
      [&] {
        for (int i = 0; i < n; i++)
          R->ctx->HMult(res[i], *static_cast<Ciphertext<word> *>(a[i]), *static_cast<Ciphertext<word> *>(b[i]),
                        key, rescale != 0);
      },
      ms);
}

int refx_time_hrot(void *p, void *a, int rot, int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx *>(p);
  Ciphertext<word> res;
  auto &A = *static_cast<Ciphertext<word> *>(a);
  const auto &key = R->ui->GetRotationKey(rot);
  return time_loop(warmup, iters, [&] { R->ctx->HRot(res, A, key, rot); }, ms);
}

// NTT then INTT of `npoly` resident polynomials over (num_main, 0, 0) per
// iteration (NTT(..., false), INTT(..., true): the round trip returns the input).
int refx_time_ntt_roundtrip(void *p, int num_main, int npoly, int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx *>(p);
  NPInfo np(num_main, 0, 0);
  size_t w = poly_words(np, R->degree);
  std::vector<DeviceVector<word>> bufs, tmps;
  for (int i = 0; i < npoly; i++) {
    bufs.emplace_back(static_cast<int>(w));
    tmps.emplace_back(static_cast<int>(w));
    cudaMemset(bufs.back().data(), 0, w * 4);
  }
  return time_loop(
      warmup, iters,
      [&] {
        for (int i = 0; i < npoly; i++) {
          DvView<word> tv = tmps[i].View();
          DvView<word> bv = bufs[i].View();
          R->ctx->ntt_handler_.NTT(tv, np, bufs[i].ConstView(), false);
          R->ctx->ntt_handler_.INTT(bv, np, tmps[i].ConstView(), true);
        }
      },
      ms);
}

int refx_time_boot(void *p, void *in, int min_ks, int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx *>(p);
  if (!R->boot) return -1;
  Ciphertext<word> res;
  auto &A = *static_cast<Ciphertext<word> *>(in);
  return time_loop(warmup, iters, [&] { R->boot->Boot(res, A, R->ui->GetEvkMap(), min_ks != 0); }, ms);
}

}  // extern "C"

// ---- the 64-bit word path (Context<uint64_t>, Context.cpp:952) ----

namespace {
using word64 = uint64_t;
struct RefCtx64 {
  std::unique_ptr<Parameter<word64>> param;
  ContextPtr<word64> ctx;
  int degree = 0;
};
void copy_in64(DeviceVector<word64> &dst, const uint64_t *src, size_t words) {
  dst.resize(static_cast<int>(words));
  cudaMemcpy(dst.data(), src, words * 8, cudaMemcpyHostToDevice);
}
void copy_out64(uint64_t *dst, const DeviceVector<word64> &src, size_t words) {
  cudaMemcpy(dst, src.data(), words * 8, cudaMemcpyDeviceToHost);
}
void ct_in64(RefCtx64 &R, Ciphertext<word64> &ct, int level, const uint64_t *bx, const uint64_t *ax) {
  NPInfo np = R.param->LevelToNP(level);
  ct.RemoveRx();
  ct.ModifyNP(np);
  ct.SetScale(R.param->GetScale(std::min(level, R.param->default_encryption_level_)));
  ct.SetNumSlots(R.degree / 2);
  const size_t w = poly_words(np, R.degree);
  copy_in64(ct.bx_, bx, w);
  copy_in64(ct.ax_, ax, w);
}
void key_in64(RefCtx64 &R, EvaluationKey<word64> &k, int beta, const uint64_t *bx, const uint64_t *ax) {
  NPInfo np(R.param->GetMaxNumMain(), R.param->GetMaxNumTer(), R.param->alpha_);
  k = EvaluationKey<word64>(np, beta);
  const size_t w = poly_words(np, R.degree);
  for (int i = 0; i < beta; i++) {
    copy_in64(k.bx_.at(i), bx + i * w, w);
    copy_in64(k.ax_.at(i), ax + i * w, w);
  }
}
}  // namespace

extern "C" {

int refx64_create(int log_degree, int log_scale, int enc_level, int n_levels, const int *level_pairs,
                  const uint64_t *main_primes, int n_main, const uint64_t *aux_primes, int n_aux,
                  const uint64_t *ter_primes, int n_ter, int add_main, int add_ter, void **out) {
  auto *R = new RefCtx64();
  std::vector<std::pair<int, int>> cfg;
  for (int i = 0; i < n_levels; i++) cfg.emplace_back(level_pairs[2 * i], level_pairs[2 * i + 1]);
  std::vector<word64> m(main_primes, main_primes + n_main), a(aux_primes, aux_primes + n_aux),
      t(ter_primes, ter_primes + n_ter);
  const double scale = static_cast<double>(UINT64_C(1) << log_scale);
  R->param = std::make_unique<Parameter<word64>>(log_degree, scale, enc_level, cfg, m, a, t,
                                                 std::make_pair(add_main, add_ter));
  R->ctx = Context<word64>::Create(*R->param);
  R->degree = R->param->degree_;
  *out = R;
  return last_cuda();
}

void refx64_destroy(void *p) {
  cudaDeviceSynchronize();
  delete static_cast<RefCtx64 *>(p);
}

int refx64_ntt(void *p, int num_main, int num_ter, int num_aux, uint64_t *data, int count, int inverse,
               int montgomery) {
  auto *R = static_cast<RefCtx64 *>(p);
  NPInfo np(num_main, num_ter, num_aux);
  const size_t w = poly_words(np, R->degree);
  DeviceVector<word64> src(static_cast<int>(w)), dst(static_cast<int>(w));
  for (int k = 0; k < count; k++) {
    cudaMemcpy(src.data(), data + k * w, w * 8, cudaMemcpyHostToDevice);
    DvView<word64> dv = dst.View(num_aux * R->degree);
    DvConstView<word64> sv = src.ConstView(num_aux * R->degree);
    if (inverse)
      R->ctx->ntt_handler_.INTT(dv, np, sv, montgomery != 0);
    else
      R->ctx->ntt_handler_.NTT(dv, np, sv, montgomery != 0);
    cudaMemcpy(data + k * w, dst.data(), w * 8, cudaMemcpyDeviceToHost);
  }
  return last_cuda();
}

int refx64_modup(void *p, int level, const uint64_t *src, uint64_t *out) {
  auto *R = static_cast<RefCtx64 *>(p);
  NPInfo np = R->param->LevelToNP(level);
  const int alpha = R->param->alpha_, q = np.GetNumQ();
  const int offset = R->param->GetMaxNumTer() - np.num_ter_;
  const int beta = DivCeil(q + offset, alpha);
  const size_t nq = static_cast<size_t>(q) * R->degree, nqp = static_cast<size_t>(q + alpha) * R->degree;
  DeviceVector<word64> s(static_cast<int>(nq));
  cudaMemcpy(s.data(), src, nq * 8, cudaMemcpyHostToDevice);
  std::vector<DeviceVector<word64>> tmp;
  std::vector<DvView<word64>> views;
  for (int i = 0; i < beta; i++) tmp.emplace_back(static_cast<int>(nqp));
  for (int i = 0; i < beta; i++) views.push_back(tmp[i].View(alpha * R->degree));
  R->ctx->mod_switch_handlers_.at(level).ModUp(views, s.ConstView());
  for (int i = 0; i < beta; i++) copy_out64(out + i * nqp, tmp[i], nqp);
  return last_cuda();
}

int refx64_moddown(void *p, int level, int kind, const uint64_t *src, uint64_t *out) {
  auto *R = static_cast<RefCtx64 *>(p);
  const int alpha = R->param->alpha_;
  NPInfo np = R->param->LevelToNP(level);
  NPInfo src_np = np;
  if (kind != 1) src_np.num_aux_ = alpha;
  NPInfo dst_np = kind == 0 ? np : R->param->LevelToNP(level - 1);
  const size_t ws = poly_words(src_np, R->degree), wd = poly_words(dst_np, R->degree);
  DeviceVector<word64> s(static_cast<int>(ws)), d(static_cast<int>(wd));
  cudaMemcpy(s.data(), src, ws * 8, cudaMemcpyHostToDevice);
  DvView<word64> dv = d.View();
  DvConstView<word64> sv = s.ConstView(src_np.num_aux_ * R->degree);
  const auto &ms = R->ctx->mod_switch_handlers_.at(level);
  if (kind == 0)
    ms.ModDown(dv, sv);
  else if (kind == 1)
    ms.Rescale(dv, sv);
  else
    ms.ModDownAndRescale(dv, sv);
  copy_out64(out, d, wd);
  return last_cuda();
}

// HMult (rescale 0/1) of two level-`level` ciphertexts with an imported key
// ([beta][L + alpha][N] per part); the result's parts go to out_bx / out_ax
// over the result level's q primes.
int refx64_hmult(void *p, int level, const uint64_t *a_bx, const uint64_t *a_ax, const uint64_t *b_bx,
                 const uint64_t *b_ax, int beta, const uint64_t *k_bx, const uint64_t *k_ax, int rescale,
                 uint64_t *out_bx, uint64_t *out_ax) {
  auto *R = static_cast<RefCtx64 *>(p);
  Ciphertext<word64> a, b, res;
  ct_in64(*R, a, level, a_bx, a_ax);
  ct_in64(*R, b, level, b_bx, b_ax);
  EvaluationKey<word64> key;
  key_in64(*R, key, beta, k_bx, k_ax);
  R->ctx->HMult(res, a, b, key, rescale != 0);
  const size_t w = poly_words(res.GetNP(), R->degree);
  copy_out64(out_bx, res.bx_, w);
  copy_out64(out_ax, res.ax_, w);
  return last_cuda();
}

int refx64_hconj(void *p, int level, const uint64_t *a_bx, const uint64_t *a_ax, int beta, const uint64_t *k_bx,
                 const uint64_t *k_ax, uint64_t *out_bx, uint64_t *out_ax) {
  auto *R = static_cast<RefCtx64 *>(p);
  Ciphertext<word64> a, res;
  ct_in64(*R, a, level, a_bx, a_ax);
  EvaluationKey<word64> key;
  key_in64(*R, key, beta, k_bx, k_ax);
  R->ctx->HConj(res, a, key);
  const size_t w = poly_words(res.GetNP(), R->degree);
  copy_out64(out_bx, res.bx_, w);
  copy_out64(out_ax, res.ax_, w);
  return last_cuda();
}

// Device time of HMult (rescale 0/1) on imported ciphertexts and key: the
// average over `iters` calls after `warmup`, CUDA events on the legacy
// stream.
int refx64_time_hmult(void *p, int level, const uint64_t *a_bx, const uint64_t *a_ax, const uint64_t *b_bx,
                      const uint64_t *b_ax, int beta, const uint64_t *k_bx, const uint64_t *k_ax, int rescale,
                      int warmup, int iters, float *ms) {
  auto *R = static_cast<RefCtx64 *>(p);
  Ciphertext<word64> a, b, res;
  ct_in64(*R, a, level, a_bx, a_ax);
  ct_in64(*R, b, level, b_bx, b_ax);
  EvaluationKey<word64> key;
  key_in64(*R, key, beta, k_bx, k_ax);
  const int rc = time_loop(warmup, iters, [&] { R->ctx->HMult(res, a, b, key, rescale != 0); }, ms);
  *ms /= iters;
  return rc;
}

// Context<uint64_t> operations by name (Context.h:101-423) on imported
// ciphertexts: a (and b) at `level`, each with rx when its rx pointer is
// given; an imported key of `beta` digits when beta > 0; arg = rotation or
// target level; (scale, value) = the constant of MultConst / AddConst,
// encoded by the reference's Encoder::EncodeConstant at `level`.  The
// result's parts go to out_bx / out_ax (and out_rx when it has rx); info =
// {num_main, num_ter, has_rx}.
int refx64_op(void *p, const char *op, int level, const uint64_t *a_bx, const uint64_t *a_ax, const uint64_t *a_rx,
              const uint64_t *b_bx, const uint64_t *b_ax, const uint64_t *b_rx, int beta, const uint64_t *k_bx,
              const uint64_t *k_ax, int arg, double scale, double value, uint64_t *out_bx, uint64_t *out_ax,
              uint64_t *out_rx, int *info) {
  auto *R = static_cast<RefCtx64 *>(p);
  Ciphertext<word64> a, b, res;
  auto load = [&](Ciphertext<word64> &c, const uint64_t *bx, const uint64_t *ax, const uint64_t *rx) {
    ct_in64(*R, c, level, bx, ax);
    if (rx) {
      c.PrepareRx();
      copy_in64(c.rx_, rx, poly_words(c.GetNP(), R->degree));
    }
  };
  load(a, a_bx, a_ax, a_rx);
  if (b_bx) load(b, b_bx, b_ax, b_rx);
  EvaluationKey<word64> key;
  if (beta > 0) key_in64(*R, key, beta, k_bx, k_ax);
  const std::string o(op);
  auto &C = *R->ctx;
  if (o == "Copy")
    C.Copy(res, a);
  else if (o == "Neg")
    C.Neg(res, a);
  else if (o == "MultImaginaryUnit")
    C.MultImaginaryUnit(res, a);
  else if (o == "Add")
    C.Add(res, a, b);
  else if (o == "Sub")
    C.Sub(res, a, b);
  else if (o == "Mult")
    C.Mult(res, a, b);
  else if (o == "Relinearize")
    C.Relinearize(res, a, key);
  else if (o == "RelinearizeRescale")
    C.RelinearizeRescale(res, a, key);
  else if (o == "MultKey")
    C.MultKey(res, a, key);
  else if (o == "Permute")
    C.Permute(res, a, arg);
  else if (o == "PermuteConjugate")
    C.PermuteConjugate(res, a);
  else if (o == "HRotAdd")
    C.HRotAdd(res, a, b, key, arg);
  else if (o == "HConjAdd")
    C.HConjAdd(res, a, b, key);
  else if (o == "LevelDown")
    C.LevelDown(res, a, arg);
  else if (o == "MultConst" || o == "AddConst") {
    Constant<word64> c;
    C.encoder_.EncodeConstant(c, level, scale, value);
    if (o == "MultConst")
      C.Mult(res, a, c);
    else
      C.Add(res, a, c);
  } else {
    return -2;
  }
  const NPInfo np = res.GetNP();
  const size_t w = poly_words(np, R->degree);
  copy_out64(out_bx, res.bx_, w);
  copy_out64(out_ax, res.ax_, w);
  if (res.HasRx() && out_rx) copy_out64(out_rx, res.rx_, w);
  info[0] = np.num_main_;
  info[1] = np.num_ter_;
  info[2] = res.HasRx() ? 1 : 0;
  return last_cuda();
}

int refx64_hrot(void *p, int level, const uint64_t *a_bx, const uint64_t *a_ax, int beta, const uint64_t *k_bx,
                const uint64_t *k_ax, int rot, uint64_t *out_bx, uint64_t *out_ax) {
  auto *R = static_cast<RefCtx64 *>(p);
  Ciphertext<word64> a, res;
  ct_in64(*R, a, level, a_bx, a_ax);
  EvaluationKey<word64> key;
  key_in64(*R, key, beta, k_bx, k_ax);
  R->ctx->HRot(res, a, key, rot);
  const size_t w = poly_words(res.GetNP(), R->degree);
  copy_out64(out_bx, res.bx_, w);
  copy_out64(out_ax, res.ax_, w);
  return last_cuda();
}

}  // extern "C"
