/*
 * cheddar_b200.h — C ABI of the B200-native CKKS evaluation core.
 *
 * Each entry point replaces one call of the reference's server-side C++ API
 * (scale-snu/cheddar-fhe); the reference interface is cited beside it.
 * Plain pointers and sizes only.  Every function returns CHD_OK (0) or an
 * error code; chd_last_error() describes the last failure of the calling
 * thread.  (The reference terminates the process on any failed assertion,
 * include/common/Assert.h:9-21; this ABI reports instead.)
 *
 * Data layout (reference include/core/Parameter.h:198-206): a polynomial is
 * [num_primes][N] uint32 residues, prime order = terminal primes reversed,
 * main primes, auxiliary primes; every residue canonical in [0, q), in the
 * bit-reversed evaluation domain and in Montgomery form (x * 2^32 mod q).
 * Evaluation keys are beta pairs (bx, ax), each over the key basis of all
 * L = main + terminal primes followed by the alpha auxiliary primes.
 * Device buffers handed to the library (wrapped ciphertexts, plaintexts, the
 * raw NTT / ModUp / ModDown / BConv operands) start on a 16-byte boundary;
 * other pointers are rejected with CHD_ERR_INVALID_ARG.
 *
 * Threading: a context is not re-entrant; all its work is ordered on one CUDA
 * stream (chd_context_set_stream).  Calls return before the GPU finishes;
 * chd_ct_export and chd_context_synchronize wait.
 */
#ifndef CHEDDAR_B200_H_
#define CHEDDAR_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHD_OK 0
#define CHD_ERR_INVALID_ARG 1
#define CHD_ERR_INVALID_LEVEL 2
#define CHD_ERR_SHAPE 3
#define CHD_ERR_CUDA 4
#define CHD_ERR_ALLOC 5
#define CHD_ERR_UNSUPPORTED 6
#define CHD_ERR_KEY 7
#define CHD_ERR_PARSE 8
#define CHD_ERR_INTERNAL 9 /* an unexpected failure inside the library (message in chd_last_error) */

/* ModDown family selector for chd_moddown_raw */
#define CHD_MODDOWN 0
#define CHD_RESCALE 1
#define CHD_MODDOWN_RESCALE 2

typedef struct chd_context chd_context;
typedef struct chd_ciphertext chd_ciphertext;
typedef struct chd_evk chd_evk;
typedef struct chd_evk_map chd_evk_map;

const char *chd_last_error(void);

/* ---- context ------------------------------------------------------------ */
/* Parameter JSON of the reference schema (unittest/Testbed.h:95-221) ->
 * Parameter(...) (include/core/Parameter.h:42-47) + Context::Create
 * (include/core/Context.h:70). */
int chd_context_create_json(const char *json_text, int device, chd_context **out);
/* Parameter(log_degree, base_scale, default_encryption_level, level_config,
 * main_primes, aux_primes, ter_primes, additional_base) + Context::Create
 * (include/core/Parameter.h:42-47, include/core/Context.h:70).
 * level_config holds num_levels (num_main, num_ter) pairs. */
int chd_context_create(int log_degree, double base_scale, int default_encryption_level,
                       const int *level_config, int num_levels, const uint32_t *main_primes,
                       int num_main, const uint32_t *aux_primes, int num_aux,
                       const uint32_t *ter_primes, int num_ter, int additional_main,
                       int additional_ter, int device, chd_context **out);
void chd_context_destroy(chd_context *ctx);
/* Orders all later work of ctx on the given cudaStream_t (NULL: the
 * context's own non-blocking stream).  No reference counterpart: the
 * reference uses the legacy default stream only (src/core/DeviceVector.cpp:68). */
int chd_context_set_stream(chd_context *ctx, void *cuda_stream);
int chd_context_synchronize(chd_context *ctx);
/* Parameter::LevelToNP (include/core/Parameter.h:184) */
int chd_level_np(const chd_context *ctx, int level, int *num_main, int *num_ter);
/* Parameter::max_level_, degree_, alpha_, L_ (include/core/Parameter.h:56-64) */
int chd_max_level(const chd_context *ctx);
int chd_degree(const chd_context *ctx);
int chd_alpha(const chd_context *ctx);
int chd_num_q_primes(const chd_context *ctx);
/* Parameter::GetScale / GetRescalePrimeProd (include/core/Parameter.h:86-100) */
double chd_scale(const chd_context *ctx, int level);
double chd_rescale_prime_prod(const chd_context *ctx, int level);
/* global index (max-level order) of every prime of an np; returns the count */
int chd_prime_gidx(const chd_context *ctx, int num_main, int num_ter, int num_aux, int *out);

/* ---- ciphertexts (include/core/Container.h:131-218) ------------------------ */
int chd_ct_create(chd_context *ctx, chd_ciphertext **out);
void chd_ct_destroy(chd_ciphertext *ct);
/* Wraps caller-owned device buffers (each words_per_part uint32 long). */
int chd_ct_wrap(chd_context *ctx, int num_main, int num_ter, int num_aux, int has_rx, double scale,
                int num_slots, uint32_t *bx, uint32_t *ax, uint32_t *rx, size_t words_per_part,
                chd_ciphertext **out);
/* Copies residues in ([num_q + num_aux][N] per part).  src_on_device: the
 * pointers are device pointers (else host). */
int chd_ct_import(chd_context *ctx, chd_ciphertext *ct, int num_main, int num_ter, int num_aux,
                  int has_rx, double scale, int num_slots, const uint32_t *bx, const uint32_t *ax,
                  const uint32_t *rx, int src_on_device);
int chd_ct_export(chd_context *ctx, const chd_ciphertext *ct, uint32_t *bx, uint32_t *ax,
                  uint32_t *rx, int dst_on_device);
/* Ciphertext::GetNP / HasRx / GetScale / GetNumSlots */
int chd_ct_info(const chd_ciphertext *ct, int *num_main, int *num_ter, int *num_aux, int *has_rx,
                double *scale, int *num_slots);
/* device pointers of the parts (valid until the ciphertext changes shape);
 * the reference exposes them as the public bx_ / ax_ / rx_ DeviceVectors
 * (include/core/Container.h:147-156) */
int chd_ct_device_ptrs(const chd_ciphertext *ct, uint32_t **bx, uint32_t **ax, uint32_t **rx);

/* ---- evaluation keys (include/core/Container.h:283-344, EvkMap.h:23-26) --- */
/* beta pairs over [L + alpha][N]: bx and ax each beta * (L+alpha) * N words */
int chd_evk_create(chd_context *ctx, int beta, const uint32_t *bx, const uint32_t *ax,
                   int src_on_device, chd_evk **out);
void chd_evk_destroy(chd_evk *evk);
/* EvaluationKey::GetBeta / GetNP (Container.h:300-312): digits and key basis */
int chd_evk_info(const chd_evk *evk, int *beta, int *num_main, int *num_ter, int *num_aux);
/* the key's beta pairs [beta][np.total][N] to host (or device) buffers, the
 * layout chd_evk_create / chd_evk_create_np take */
int chd_evk_export(chd_context *ctx, const chd_evk *evk, uint32_t *bx, uint32_t *ax, int dst_on_device);

/* ---- evaluator (include/core/Context.h:101-423) ----------------------------- */
/* Context::Add / Sub / Neg (Context.cpp:146-169, 205-229, 306-315) */
int chd_add(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b);
int chd_sub(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b);
int chd_neg(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* Context::Mult(Ct, Ct, Ct): tensor product, result carries rx */
int chd_mult(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b);
/* Context::Mult(Ct, Ct, Const) / Add(Ct, Ct, Const): cx = one Montgomery word
 * per prime of a's np (host pointer) */
int chd_mult_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a,
                   const uint32_t *cx, double const_scale);
int chd_add_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx);
/* Context::Mult(Ct, Ct, Pt): pt_dev = [num_q][N] device residues */
int chd_mult_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a,
                   const uint32_t *pt_dev, double pt_scale);
/* Context::MultImaginaryUnit (Context.cpp:550-560) */
int chd_mult_imaginary_unit(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* Context::Rescale (Context.cpp:740-775) */
int chd_rescale(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* Context::Relinearize / RelinearizeRescale (Context.cpp:562-565, 715-738) */
int chd_relinearize(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *key);
int chd_relinearize_rescale(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a,
                            const chd_evk *key);
/* Context::MultKey (Context.cpp:585-608) */
int chd_mult_key(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *key);
/* Context::HMult(res, a, b, mult_key, rescale) (Context.cpp:862-871) */
int chd_hmult(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a,
              const chd_ciphertext *b, const chd_evk *mult_key, int rescale);
/* Batched HMult over count independent pairs (no reference counterpart; the
 * reference exposes one HMult per call).  Pairs at different levels run as
 * one batched pipeline per level. */
int chd_hmult_batch(chd_context *ctx, int count, chd_ciphertext *const *res,
                    const chd_ciphertext *const *a, const chd_ciphertext *const *b,
                    const chd_evk *mult_key, int rescale);
/* Context::Copy (Context.cpp:132-143) */
int chd_copy(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* Context::MultUnsafe(Ct, Ct, Ct, level) (Context.cpp:370-412): tensor
 * product at `level` (-1: the lower input level), reading each input past
 * its extra terminal primes; result carries rx.  Inputs without rx or aux. */
int chd_mult_unsafe(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
                    int level);
/* Context::MultUnsafe(Ct, Ct, Const, level) (Context.cpp:458-500): cx = the
 * constant's Montgomery residues over the q primes of const_level (as
 * chd_encode_const writes them), const_scale its scale; result at `level`
 * (-1: the lower of the two levels). */
int chd_mult_unsafe_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx,
                          int const_level, double const_scale, int level);
/* Context::MadUnsafe (Context.cpp:873-915): res += a * const over res's
 * primes; res's scale must equal a's times const_scale, the slot counts
 * match, res gains a zero rx when a has one. */
int chd_mad_unsafe(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx,
                   int const_level, double const_scale);
/* Context::Permute / PermuteConjugate (Context.cpp:502-547): the automorphism
 * alone (use after chd_mult_key); rotation by 0 copies. */
int chd_permute(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, int rot_dist);
int chd_permute_conjugate(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* Context::HConjAdd (Context.cpp:836-860): res = HConj(a) + b */
int chd_hconj_add(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
                  const chd_evk *conj_key);
/* Context::LevelDown (Context.cpp:917-929): per level, times the constant 1
 * at that level's scale, then Rescale, down to target_level */
int chd_level_down(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, int target_level);
/* Context::MultKeyNoModDown(Ct, Ct, Evk) (Context.cpp:650-700): the
 * key switch of a left in the extended basis Q u P; with rx (relinearisation):
 * ModUp(rx) (.) key + P * (bx, ax); chd_moddown finishes it.  Without rx
 * (a rotation's key switch): ModUp(ax) (.) key + (P * bx, 0). */
int chd_mult_key_no_moddown(chd_context *ctx, chd_ciphertext *accum, const chd_ciphertext *a, const chd_evk *key);
/* Context::IsMultUnsafeCompatible (Context.cpp:357-368): 1 / 0, -1 for a
 * null context or a level out of range */
int chd_mult_unsafe_compatible(const chd_context *ctx, int level1, int level2);
/* Context::Add(Ct, Ct, Pt) / Sub(Ct, Ct, Pt) (Context.cpp:171-186,
 * 231-246): res.bx = a.bx +/- pt, ax and rx copied; pt_dev = [num_q + num_aux
 * of a][N] device residues, pt_scale must equal a's scale (relative 1e-12). */
int chd_add_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                  double pt_scale);
int chd_sub_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                  double pt_scale);
/* Context::Sub(Ct, Ct, Const) (Context.cpp:248-263): res.bx = a.bx - c */
int chd_sub_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx);
/* Context::Sub(Ct, Pt, Ct) / Sub(Ct, Const, Ct) (Context.cpp:265-304):
 * res = pt - b (c - b): bx = pt - b.bx, ax = -b.ax, rx = -b.rx; the
 * plaintext's / constant's scale must equal b's and becomes res's. */
int chd_sub_plain_ct(chd_context *ctx, chd_ciphertext *res, const uint32_t *pt_dev, double pt_scale,
                     const chd_ciphertext *b);
int chd_sub_const_ct(chd_context *ctx, chd_ciphertext *res, const uint32_t *cx, double const_scale,
                     const chd_ciphertext *b);
/* Context::MultUnsafe(Ct, Ct, Pt, level) (Context.cpp:414-456): pt_dev =
 * [num_q(pt_level) + pt_num_aux][N] (as chd_encode writes it); result at
 * `level` (-1: the lower level) with the fewer aux primes of the two, both
 * read past their extra terminal primes. */
int chd_mult_unsafe_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                          int pt_level, int pt_num_aux, double pt_scale, int level);

/* Context::HRot / HConj / HRotAdd (Context.cpp:776-830) */
int chd_hrot(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *rot_key,
             int rot_dist);
int chd_hconj(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *conj_key);
int chd_hrot_add(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a,
                 const chd_ciphertext *b, const chd_evk *rot_key, int rot_dist);
/* HoistHandler::EvaluateBabyStep with the fused key-mult
 * (src/extension/Hoist.cu:578-691): count rotations of a in one launch,
 * results left in the extended basis (num_aux = alpha). */
int chd_hoisted_rotate(chd_context *ctx, const chd_ciphertext *a, int count, const int *rot_dists,
                       const chd_evk *const *rot_keys, chd_ciphertext *const *out);
/* ModSwitchHandler::ModDown of an extended-basis ciphertext (ModSwitch.cu:511-527) */
int chd_moddown(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a);
/* ModDown of `count` ciphertexts at one level (Q u P -> Q), e.g. the
 * rotations of one hoisted set, through one fused pipeline: the same
 * residues as chd_moddown on each (no reference counterpart; the reference
 * keeps hoisted rotations in Q u P and reduces them one accumulation at a
 * time, Hoist.cu:695-975). */
int chd_moddown_batch(chd_context *ctx, int count, chd_ciphertext *const *res, const chd_ciphertext *const *a);

/* ---- raw kernels on device buffers (parity entry points) -------------------- */
/* NTTHandler::NTT / INTT (include/core/NTT.h:55-62): count consecutive
 * polynomials of np, in place. */
int chd_ntt(chd_context *ctx, int num_main, int num_ter, int num_aux, uint32_t *data_dev, int mont,
            int count);
int chd_intt(chd_context *ctx, int num_main, int num_ter, int num_aux, uint32_t *data_dev, int mont,
             int count);
/* ModSwitchHandler::ModUp (ModSwitch.cu:429-509): src [num_q][N] ->
 * dst [beta][num_q + alpha][N] */
int chd_modup_raw(chd_context *ctx, int level, const uint32_t *src_dev, uint32_t *dst_dev);
/* ModSwitchHandler::ModDown / Rescale / ModDownAndRescale (ModSwitch.cu:511-564)
 * on npoly consecutive polynomials */
int chd_moddown_raw(chd_context *ctx, int level, int type, const uint32_t *src_dev, uint32_t *dst_dev,
                    int npoly);
/* kernel::ModSwitchMatrixMult (ModSwitch.cu:23-171): K centred source limbs
 * (global prime indices src_gidx) -> M limbs (dst_gidx), table
 * T[m][k] = centre(prod_{j != k} src_j * 2^64 mod dst_m). */
int chd_bconv_raw(chd_context *ctx, const int32_t *xt_dev, const int *src_gidx, int K,
                  const int *dst_gidx, int M, uint32_t *out_dev);

/* ---- bootstrapping building blocks ---- */
/* Encoder::Encode (src/core/Encode.cpp:23-41, 84-107, 135-190): msg_len
 * complex slots (re, im; padded to a power of two, written to *num_slots)
 * at `scale` -> plaintext [num_q(level) + num_aux][N] at pt_dev, evaluation
 * domain, Montgomery form (prime order: terminal reversed, main, aux).
 * On the device: FP64 special IFFT, truncation toward zero, residues, NTT;
 * returns when the plaintext is written. */
int chd_encode(chd_context *ctx, int level, double scale, const double *re, const double *im, int msg_len,
               int num_aux, uint32_t *pt_dev, int *num_slots);
/* Encoder::Decode (src/core/Encode.cpp:45-70, 109-133, 192-248): plaintext
 * [num_q(level)][N] at pt_dev (evaluation domain, Montgomery form, no aux
 * primes) at `scale` -> num_slots complex slots (a power of two <= N/2)
 * written to the host arrays re, im.  On the device: INTT times
 * (N q-hat)^-1, CRT to the centred integer (exact while its magnitude is
 * below 2^127), double / scale, FP64 special FFT; the same doubles as the
 * reference's decoder.  Returns when the slots are written. */
int chd_decode(chd_context *ctx, int level, double scale, const uint32_t *pt_dev, int num_slots, double *re,
               double *im);
/* Encoder::EncodeConstant (Encode.cpp:250-275): cx[num_q(level) + num_aux]
 * Montgomery residues of trunc(value * scale), host memory. */
int chd_encode_const(chd_context *ctx, int level, double scale, double value, int num_aux, uint32_t *cx);
/* BootContext::ModUpToMax (src/extension/BootContext.cpp:186-270): a at
 * level -1 -> res at the top level.  With sparse-secret encapsulation (the
 * parameters' dense Hamming weight above the sparse one) the key map must
 * hold the dense-to-sparse and sparse-to-dense keys; otherwise keys may be
 * NULL. */
int chd_modup_to_max(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk_map *keys);

/* EvkMap (include/core/EvkMap.h): rotation / conjugation / multiplication
 * keys by index.  The map borrows the keys; they must outlive it. */
int chd_evk_map_create(chd_context *ctx, chd_evk_map **out);
void chd_evk_map_destroy(chd_evk_map *m);
int chd_evk_map_set_rotation(chd_evk_map *m, int rot_idx, const chd_evk *key);
int chd_evk_map_set_conjugation(chd_evk_map *m, const chd_evk *key);
int chd_evk_map_set_mult(chd_evk_map *m, const chd_evk *key);
/* EvkMap::GetDenseToSparseKey / GetSparseToDenseKey (sparse-secret
 * encapsulation, UserInterface.cu:342-356): the dense-to-sparse key over the
 * level -1 primes and as many aux primes (one digit, chd_evk_create_np), the
 * sparse-to-dense key over the full key basis (its digit 0 is used). */
int chd_evk_map_set_dense_to_sparse(chd_evk_map *m, const chd_evk *key);
int chd_evk_map_set_sparse_to_dense(chd_evk_map *m, const chd_evk *key);
/* An evaluation key over an explicit basis (num_main, num_ter, num_aux):
 * beta digits of [num_main + num_ter + num_aux][N] per part. */
int chd_evk_create_np(chd_context *ctx, int num_main, int num_ter, int num_aux, int beta, const uint32_t *bx,
                      const uint32_t *ax, int src_on_device, chd_evk **out);

/* LinearTransform (src/extension/LinearTransform.cpp:77-124) with the
 * HoistHandler's double-hoisted baby-step / giant-step evaluation
 * (src/extension/Hoist.cu).  The matrix has `width` slots and n_diag
 * diagonals diag_idx[i] with values re/im [n_diag][width]
 * (d[k] = M[k][(k + i) mod width]); diagonals are encoded at pt_level /
 * pt_scale with the alpha auxiliary primes.  Evaluation: res (level
 * pt_level - 1, scale pt_scale * in.scale / rescale prime product) = M in. */
typedef struct chd_lintrans chd_lintrans;
int chd_lintrans_create(chd_context *ctx, int width, int n_diag, const int *diag_idx, const double *re,
                        const double *im, int pt_level, double pt_scale, int bs, int gs, int pre_rotation,
                        int additional_pt_rot, chd_lintrans **out);
void chd_lintrans_destroy(chd_lintrans *lt);
/* HoistHandler::AddRequiredRotations: the rotation keys the transform uses
 * (min_ks != 0: only the baby and giant strides) */
int chd_lintrans_rotations(const chd_lintrans *lt, int min_ks, int *out, int cap, int *count);
/* the compiled plaintext map (giant step, baby step, message [width]) */
int chd_lintrans_num_pts(const chd_lintrans *lt, int *count);
int chd_lintrans_pt(const chd_lintrans *lt, int i, int *gs, int *bs, double *re, double *im);
/* min_ks != 0: the min-KS evaluation (HoistHandler::EvaluateMinKS*,
 * Hoist.cu:490-552): repeated rotations by the strides, in the Q basis */
int chd_lintrans_evaluate(chd_context *ctx, const chd_lintrans *lt, chd_ciphertext *res, const chd_ciphertext *in,
                          const chd_evk_map *keys, int min_ks);

/* Compiled ciphertext programs: EvalPoly (src/extension/EvalPoly.cpp) of
 * a polynomial given by its coefficients (Chebyshev basis when chebyshev
 * != 0) for an input at (input_level, input_scale), result at
 * target_scale; and EvalMod (src/extension/EvalMod.cpp: x - 1/(4K), the
 * Chebyshev cosine of coeffs, num_double_angle double-angle steps) for an
 * input at start_level.  Running a program needs the multiplication key in
 * the key map.  chd_program_json writes the compiled op list (ops,
 * registers, constants as (level, scale, value)) for inspection and
 * testing; *len receives the size including the terminating zero. */
typedef struct chd_program chd_program;
int chd_poly_create(chd_context *ctx, const double *coeffs, int n, int input_level, double input_scale,
                    double target_scale, int chebyshev, chd_program **out);
int chd_evalmod_create(chd_context *ctx, int start_level, const double *coeffs, int n, int num_double_angle,
                       int initial_K, chd_program **out, double *start_scale, double *end_scale);
void chd_program_destroy(chd_program *p);
/* BootParameter's EvalMod Chebyshev coefficients (BootParameter.cpp:13-23);
 * returns their number, copies up to cap of them */
int chd_boot_mod_coefficients(double *out, int cap);
int chd_program_json(const chd_program *p, char *buf, size_t cap, size_t *len);
int chd_program_run(chd_context *ctx, const chd_program *p, chd_ciphertext *res, const chd_ciphertext *in,
                    const chd_evk_map *keys);

/* BootContext (src/extension/BootContext.cpp) for one slot count:
 * PrepareEvalMod + PrepareEvalSpecialFFT (EvalSpecialFFT.cpp) with
 * num_cts_levels / num_stc_levels (BootParameter; log_message_ratio 5 in
 * the reference), then Boot (full slots, BootVariant::kNormal, with
 * sparse-secret encapsulation when the parameters' dense Hamming weight
 * exceeds the sparse one): in at a level in [0, default encryption level]
 * (brought to level 0 by LevelDown) -> res at the end level (StC start -
 * num_stc_levels).  Keys: the multiplication and conjugation keys, every
 * rotation chd_boot_rotations lists, and with encapsulation the
 * dense-to-sparse and sparse-to-dense keys.
 * chd_boot_levels: {CtS start, EvalMod start, StC start, end level,
 * log2 scale-up} and {CtS constant, StC constant, EvalMod start scale,
 * EvalMod end scale, final scale}.  chd_boot_json / _lt_info / _lt_pt
 * export the compiled program and the transforms' plaintext maps. */
typedef struct chd_boot chd_boot;
int chd_boot_create(chd_context *ctx, int num_slots, int num_cts_levels, int num_stc_levels, int log_message_ratio,
                    chd_boot **out);
/* PrepareEvalSpecialFFT(num_slots, variant) (BootContext.h:16-20, 96-97):
 * num_slots a power of two from 256 to N/2 (below N/2: Trace after
 * ModUpToMax, extended 2n x 2n CtS / StC phases, one EvalMod on both parts,
 * a final HRotAdd by n); variant CHD_BOOT_NORMAL, CHD_BOOT_IMAGINARY_REMOVING
 * (StC constant / 2 and res = HConj(res) + res at the end: a real result) or
 * CHD_BOOT_MERGE_TWO_REAL (StC constant / 2; the caller combines two real
 * inputs before and after).  chd_boot_create is variant CHD_BOOT_NORMAL. */
#define CHD_BOOT_NORMAL 0
#define CHD_BOOT_IMAGINARY_REMOVING 1
#define CHD_BOOT_MERGE_TWO_REAL 2
int chd_boot_create_variant(chd_context *ctx, int num_slots, int variant, int num_cts_levels, int num_stc_levels,
                            int log_message_ratio, chd_boot **out);
void chd_boot_destroy(chd_boot *b);
int chd_boot_rotations(const chd_boot *b, int min_ks, int *out, int cap, int *count);
int chd_boot_levels(const chd_boot *b, int *levels, double *scales);
/* (no counterpart: exports of the compiled plan -- op program, linear
 * transforms and their plaintexts -- for checkers) */
int chd_boot_json(const chd_boot *b, char *buf, size_t cap, size_t *len);
int chd_boot_lt_info(const chd_boot *b, int i, int *level, double *scale, int *npts, int *width);
int chd_boot_lt_pt(const chd_boot *b, int i, int j, int *gs, int *bs, double *re, double *im);
/* Boot(res, input, evk_map, min_ks) (BootContext.h:139-140) */
int chd_boot_run(chd_context *ctx, chd_boot *b, chd_ciphertext *res, const chd_ciphertext *in, const chd_evk_map *keys,
                 int min_ks);
/* Boot of `count` ciphertexts in one call (no reference counterpart; the
 * reference bootstraps one ciphertext per call): every key switch, rescale
 * and linear transform of the bootstrapping program runs once over the
 * whole batch.  Each res[i] equals chd_boot_run(res[i], in[i]); results must
 * be distinct (a result may alias an input).  Inputs may sit at different
 * levels (each is brought down to level 0 first). */
int chd_boot_run_batch(chd_context *ctx, chd_boot *b, int count, chd_ciphertext *const *res,
                       const chd_ciphertext *const *in, const chd_evk_map *keys, int min_ks);

/* CUDA graphs of library calls (no reference counterpart; the reference
 * issues every kernel from the host).  chd_graph_begin starts capturing the
 * GPU work of the following calls on the context stream; chd_graph_end
 * instantiates it; chd_graph_launch replays it on the context stream,
 * reading and writing the same buffers.  Calls made while capturing must
 * not allocate or wait: run the same calls once before capturing so that
 * results and scratch are already sized. */
typedef struct chd_graph chd_graph;
int chd_graph_begin(chd_context *ctx);
int chd_graph_end(chd_context *ctx, chd_graph **out);
int chd_graph_launch(chd_context *ctx, const chd_graph *g);
void chd_graph_destroy(chd_graph *g);

/* Batched kernel::ModSwitchMatrixMult: npoly polynomials, each K centred
 * source limbs [K][N] (xt_dev + i*K*N) -> M limbs [M][N] (out_dev + i*M*N),
 * same table and result as chd_bconv_raw.  engine CHD_BCONV_CUDA_CORE runs
 * int64 multiply-adds; CHD_BCONV_TENSOR_CORE runs the contraction as an INT8
 * 4-limb GEMM on the tcgen05 tensor cores with int32 accumulation (exact,
 * bit-identical output).  Asynchronous; chd_context_synchronize reports a
 * tensor-core wait that ran out. */
#define CHD_BCONV_CUDA_CORE 0
#define CHD_BCONV_TENSOR_CORE 1
#define CHD_BCONV_AUTO 2 /* chd_set_ks_engine only: autotuned per launch shape */
/* chd_set_ks_engine only: the tensor-core column pass on 256-thread tiles
 * (8 coefficients per thread, twice the warps per SM) for ModUp / ModDown
 * with at most 12 sources; larger ones use CHD_BCONV_TENSOR_CORE */
#define CHD_BCONV_TENSOR_CORE_WIDE 3
int chd_bconv_batch(chd_context *ctx, int engine, int npoly, const int32_t *xt_dev, const int *src_gidx, int K,
                    const int *dst_gidx, int M, uint32_t *out_dev);

/* Engine of the base conversion inside every ModUp / ModDown of the fused
 * key-switching, rescaling and bootstrapping paths (HMult, relinearize,
 * rotations, hoisted rotations, linear transforms, ModDown epilogues):
 * CHD_BCONV_CUDA_CORE (int64 multiply-adds), CHD_BCONV_TENSOR_CORE (the
 * column pass issues INT8 byte-limb MMAs on the tcgen05 tensor cores with
 * int32 accumulation in TMEM, 128-thread tiles) or
 * CHD_BCONV_TENSOR_CORE_WIDE (the same on 256-thread tiles).  All give
 * bit-identical residues.
 * CHD_BCONV_AUTO autotunes: the first column pass of each launch shape
 * (device, sources, jobs, targets) outside a stream capture times the
 * three with each split of the targets over 1, 2, 4 or the heuristic
 * number of CTAs per column tile (one host synchronisation per shape and
 * process) and keeps the fastest (a tensor-core candidate within 3 % of a
 * faster CUDA-core one, as it shares an SM better with the other stream's
 * kernels); an untuned shape met during a capture
 * uses the tensor cores with the heuristic split.  No reference counterpart (the reference has one CUDA-core
 * implementation, src/core/ModSwitch.cu:23-171).  chd_get_ks_engine returns
 * the engine, -1 for a null context. */
int chd_set_ks_engine(chd_context *ctx, int engine);
int chd_get_ks_engine(const chd_context *ctx);
/* The autotuner's choices so far (no reference counterpart): per launch
 * shape six ints (device, largest source count K, jobs, largest target
 * count M, engine: 0 CUDA cores, 1 tensor cores, 3 / 4 tensor cores on
 * 256-thread tiles at 80 / 128 registers, target split) into out
 * (capacity cap shapes);
 * returns the number of shapes tuned in this process. */
int chd_ks_tuned_shapes(int *out, int cap);
/* The same for the key-switch row pass (no reference counterpart): with
 * CHD_BCONV_AUTO its first launch of each shape times the variant that
 * loads each digit's key words and the next digit's ModUp row ahead (2 CTAs
 * per SM) against the one that loads where it computes at 3 and at 4 CTAs
 * per SM; five ints per shape (device, ciphertexts, largest row count of
 * the launch, mode, variant: 0 loads where used at 3 CTAs per SM, 1 loads
 * ahead, 2 loads where used at 4); returns the count. */
int chd_ks_rows_tuned_shapes(int *out, int cap);
/* Two-stream key switching (no reference counterpart; on by default, the
 * environment variable CHD_SPLIT_STREAMS=0 turns it off at context
 * creation): a fused key switch of two or more ciphertexts, a batched ModUp
 * of two or more, and a ModDown family call on four or more polynomials, at
 * N = 2^16 (HMult / Relinearize / MultKey / HRot batches, hoisted rotation
 * batches, batched ModDown and rescaling, batched bootstrapping) runs its
 * two halves on the context stream and on a second
 * stream of the context, forked from and joined back into the context
 * stream by events (graph capture included), unless a result of one half is
 * an operand or a result of the other.  Results are identical either way.
 * With the stage timer on (chd_stage_timing) each half's spans are recorded
 * on its own stream: the launch counts are the split pipeline's, the summed
 * times those of kernels that overlap (time the one-stream pipeline for
 * per-kernel figures).  chd_get_stream_split returns 1 / 0, or -1 for a null
 * context. */
int chd_set_stream_split(chd_context *ctx, int on);
int chd_get_stream_split(const chd_context *ctx);

/* ---- residue serialization (no counterpart in the reference, whose objects
 * live only in device memory): a ciphertext or key as a self-describing
 * byte buffer (magic, ring degree, prime counts, scale and slot count,
 * the primes of its rows, then the residues in their device layout).
 * Loading checks the degree and every prime against the context.  With buf
 * null, *len receives the size needed. ---- */
int chd_ct_serialize(chd_context *ctx, const chd_ciphertext *ct, void *buf, size_t cap, size_t *len);
int chd_ct_deserialize(chd_context *ctx, chd_ciphertext *ct, const void *buf, size_t len);
int chd_evk_serialize(chd_context *ctx, const chd_evk *evk, void *buf, size_t cap, size_t *len);
int chd_evk_deserialize(chd_context *ctx, const void *buf, size_t len, chd_evk **out);

/* ---- test-only client (the reference's UserInterface, src/UserInterface.cu:
 * 110-541, "not secure, for testing"): secrets, evaluation keys, encryption
 * and decryption on the device, reproducible from a seed.  The key and
 * ciphertext structure is the reference's; the randomness is a seeded
 * counter-based generator (the reference draws from an unseeded
 * std::random_device / mt19937_64), errors with the reference's
 * distribution, round(N(0, 3.2^2)) clamped at 6 sigma. ---- */
typedef struct chd_client chd_client;
/* UserInterface constructor (PrepareSecrets, UserInterface.cu:224-276): the
 * dense ternary secret (the parameters' dense Hamming weight, N/2 when
 * unset) and, with sparse-secret encapsulation, the sparse one, over the
 * full key basis in the NTT Montgomery domain. */
int chd_client_create(chd_context *ctx, uint64_t seed, chd_client **out);
void chd_client_destroy(chd_client *cl);
/* the secret's residues [L + alpha][N] (NTT Montgomery domain) to host
 * memory; sparse != 0 for the sparse secret (tests only) */
int chd_client_secret(chd_context *ctx, const chd_client *cl, int sparse, uint32_t *out);
/* PrepareBasicEvks / PrepareRotationKey (UserInterface.cu:278-364): keys
 * over the max-level key basis (beta digits) as chd_evk objects */
int chd_client_mult_key(chd_context *ctx, chd_client *cl, chd_evk **out);
int chd_client_rotation_key(chd_context *ctx, chd_client *cl, int rot_idx, chd_evk **out);
int chd_client_conjugation_key(chd_context *ctx, chd_client *cl, chd_evk **out);
/* sparse-secret encapsulation keys: dense-to-sparse over the level -1 primes
 * and as many aux primes, sparse-to-dense as one digit over the key basis
 * (UserInterface.cu:335-352), for chd_evk_map_set_dense_to_sparse /
 * _sparse_to_dense */
int chd_client_sse_keys(chd_context *ctx, chd_client *cl, chd_evk **dense_to_sparse, chd_evk **sparse_to_dense);
/* UserInterface::Encrypt (UserInterface.cu:132-183): plaintext
 * [num_q(level)][N] at pt_dev (as chd_encode writes it) -> ct at `level`
 * with `scale` and `num_slots`; `nonce` selects the encryption randomness. */
int chd_client_encrypt(chd_context *ctx, chd_client *cl, uint64_t nonce, int level, double scale, int num_slots,
                       const uint32_t *pt_dev, chd_ciphertext *ct);
/* UserInterface::Decrypt (UserInterface.cu:185-206): ct (relinearised, no
 * aux primes) -> plaintext [num_q][N] at pt_dev, for chd_decode. */
int chd_client_decrypt(chd_context *ctx, const chd_client *cl, const chd_ciphertext *ct, uint32_t *pt_dev);

/* Test hook for the bounded waits of the tensor-core kernels (no reference
 * counterpart: the reference's kernels have no tensor-core waits).  With
 * polls > 0 every later stand-alone tensor-core base conversion
 * (chd_bconv_batch, engine 1) makes each CTA's first accumulator wait poll an
 * mbarrier that nothing signals, `polls` times: the wait runs out, the
 * kernel records the failure in the context's device error word, waits
 * (bounded) for its MMAs in flight, releases its tensor memory and returns,
 * and the next chd_context_synchronize reports CHD_ERR_CUDA.  Outputs of
 * such launches are undefined.  polls = 0 (the default) restores normal
 * operation. */
int chd_debug_stall_tensor_waits(chd_context *ctx, int polls);

/* ModUp like chd_modup_raw, but allocating no device memory: for callers
 * that must not allocate once running (latency-critical servers, where a
 * cudaMalloc can synchronise the device; hosts whose device memory belongs
 * to another allocator or a fixed budget).  No counterpart in the reference.
 * Its scratch is one static device array of 2^21 words (8 MiB) per GPU,
 * held until the process exits: num_q(level) * N must fit (32 q primes at
 * N = 2^16), else CHD_ERR_UNSUPPORTED.  All calls share that array, so calls
 * whose GPU work overlaps race.  The first call on a device looks up the
 * array's address; make it before any stream capture. */
int chd_modup_raw_noalloc(chd_context *ctx, int level, const uint32_t *src_dev, uint32_t *dst_dev);

/* Device timing of the fused key-switch stages (no reference counterpart;
 * the reference's unit tests time whole operations, unittest/Testbed.h:24-47).
 * enable != 0 clears earlier records and starts recording CUDA events on the
 * context stream around every stage; 0 stops.  chd_stage_times waits for the
 * recorded work and returns, per stage, the summed device milliseconds and
 * the number of kernel launches:
 *   0 ModUp INTT row phase, 1 ModUp column pass, 2 key-switch row pass,
 *   3 ModDown column pass, 4 NTT row phase with the ModDown epilogue. */
#define CHD_KS_STAGES 5
int chd_stage_timing(chd_context *ctx, int enable);
int chd_stage_times(chd_context *ctx, double *ms, int *launches);

/* Host-side ModSwitch constants of one level, computed without a GPU
 * (ModSwitchHandler ctor, src/core/ModSwitch.cu:175-411).  kind: 0 = ModUp
 * digit `digit`, 1 = ModDown, 2 = Rescale, 3 = ModDownAndRescale.  Outputs:
 * c1[K] (plain (N q-hat)^-1 x restore), table[M*K] (centred BConv table),
 * inv[M] and pad[dims[2]] (Montgomery epilogue constants); dims = {K, M,
 * pad_len, restore_start, restore_end, beta}.  Buffers: c1 >= 16,
 * table >= 64*16, inv/pad >= 64 words. */
int chd_params_level_consts(const char *json_text, int level, int kind, int digit, uint32_t *c1,
                            int32_t *table, uint32_t *inv, uint32_t *pad, int *dims);

/* ---- the 64-bit word path: the reference's Context<uint64_t>
 * (src/core/NTT.cu:1313, ModSwitch.cu:688, ElementWise.cu:1706,
 * Context.cpp:952) for parameter files with primes up to 2^62, e.g.
 * parameters/bootparam_40_64bit.json.  Residues are uint64_t words in the
 * reference's layout ([num_primes][N], Montgomery form x 2^64 mod q,
 * bit-reversed evaluation domain).  N = 2^16; the evaluation core: NTT,
 * ModUp / ModDown / Rescale / ModDownAndRescale, HMult (relinearised,
 * optionally rescaled), HRot, HConj and the Context operations below.
 * Same status codes; chd_last_error describes failures. ---- */
typedef struct chd64_context chd64_context;
typedef struct chd64_ciphertext chd64_ciphertext;
typedef struct chd64_evk chd64_evk;
/* Parameter(...) + Context<uint64_t>::Create from the reference's JSON
 * schema (unittest/Testbed.h:95-221); primes are read as exact integers */
int chd64_context_create_json(const char *json, int device, chd64_context **out);
void chd64_context_destroy(chd64_context *ctx);
int chd64_context_synchronize(chd64_context *ctx);
/* work of the context on the caller's stream (NULL: back to its own) */
int chd64_context_set_stream(chd64_context *ctx, void *cuda_stream);
int chd64_max_level(const chd64_context *ctx);
int chd64_alpha(const chd64_context *ctx);
int chd64_level_np(const chd64_context *ctx, int level, int *num_main, int *num_ter);
/* the primes in global order (terminal reversed, main, auxiliary); returns
 * their count, writing at most cap */
int chd64_primes(const chd64_context *ctx, uint64_t *out, int cap);
/* NTTHandler<uint64_t>::NTT / INTT (NTT.cu:606-741): count polynomials of
 * [num_main + num_ter + num_aux][N] at data_dev, in place; mont != 0 converts
 * into (NTT) or out of (INTT) the Montgomery form */
int chd64_ntt(chd64_context *ctx, int num_main, int num_ter, int num_aux, uint64_t *data_dev, int count, int inverse,
              int mont);
/* ModSwitchHandler<uint64_t>::ModUp (ModSwitch.cu:429-509): [num_q][N] ->
 * beta x [num_q + alpha][N] */
int chd64_modup_raw(chd64_context *ctx, int level, const uint64_t *src_dev, uint64_t *dst_dev);
/* ModDown / Rescale / ModDownAndRescale (ModSwitch.cu:511-684) of npoly
 * polynomials, type CHD_MODDOWN, CHD_RESCALE or CHD_MODDOWN_RESCALE */
int chd64_moddown_raw(chd64_context *ctx, int level, int type, const uint64_t *src_dev, uint64_t *dst_dev, int npoly);
int chd64_ct_create(chd64_context *ctx, chd64_ciphertext **out);
void chd64_ct_destroy(chd64_ciphertext *ct);
/* bx, ax: [num_q(level)][N] each, host or device memory */
int chd64_ct_import(chd64_context *ctx, chd64_ciphertext *ct, int level, double scale, int num_slots,
                    const uint64_t *bx, const uint64_t *ax, int src_on_device);
int chd64_ct_export(chd64_context *ctx, const chd64_ciphertext *ct, uint64_t *bx, uint64_t *ax);
int chd64_ct_info(const chd64_ciphertext *ct, int *num_main, int *num_ter, double *scale, int *num_slots);
/* EvaluationKey<uint64_t>: beta digits over the max-level key basis,
 * [beta][L + alpha][N] each for bx and ax */
int chd64_evk_create(chd64_context *ctx, int beta, const uint64_t *bx, const uint64_t *ax, int src_on_device,
                     chd64_evk **out);
void chd64_evk_destroy(chd64_evk *key);
/* Context<uint64_t>::HMult (Context.cpp:862-871), HRot (:776-791), Rescale
 * (:739-774); the result must not alias an operand */
int chd64_hmult(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
                const chd64_evk *key, int rescale);
int chd64_hrot(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key, int rot);
/* Context<uint64_t>::HConj (Context.cpp:793-798) with a conjugation key */
int chd64_hconj(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key);
int chd64_rescale(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a);
/* The third part (rx, [num_q][N]) of an unrelinearised ciphertext: set
 * after chd64_ct_import, read back, and whether a ciphertext has one (1 /
 * 0, -1 for null) */
int chd64_ct_set_rx(chd64_context *ctx, chd64_ciphertext *ct, const uint64_t *rx, int src_on_device);
int chd64_ct_export_rx(chd64_context *ctx, const chd64_ciphertext *ct, uint64_t *rx);
int chd64_ct_has_rx(const chd64_ciphertext *ct);
/* Parameter::GetScale (Parameter.cu:145-190) for level 0 .. the default
 * encryption level, 0 otherwise */
double chd64_scale(const chd64_context *ctx, int level);
/* Encoder<uint64_t>::EncodeConstant (Encode.cpp:250-275): value x scale,
 * rounded toward zero, as one Montgomery word per prime of
 * level_np(level, num_aux) into cx */
int chd64_encode_const(chd64_context *ctx, int level, double scale, double value, int num_aux, uint64_t *cx);
/* Context<uint64_t> operations (Context.h:101-423 with word = uint64_t),
 * same meaning as their 32-bit chd_* counterparts: Copy, Neg,
 * MultImaginaryUnit (ElementWise.cu:625-658), Add / Sub (rx kept from the
 * side that has it; Context.cpp:145-229), Mult (the three-part tensor,
 * Context.cpp:316-330), Relinearize / RelinearizeRescale (rescale != 0),
 * MultKey, Permute / PermuteConjugate (conjugate != 0), HRotAdd, HConjAdd,
 * Mult / Add by a constant (one Montgomery word per prime of a's basis,
 * host memory; the constant's scale multiplies a's) and LevelDown (to
 * target_level, inputs up to the default encryption level) */
int chd64_copy(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a);
int chd64_neg(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a);
int chd64_mult_imaginary_unit(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a);
int chd64_add(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b);
int chd64_sub(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b);
int chd64_mult(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b);
int chd64_relinearize(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key,
                      int rescale);
int chd64_mult_key(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key);
int chd64_permute(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, int rot, int conjugate);
int chd64_hrot_add(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
                   const chd64_evk *key, int rot);
int chd64_hconj_add(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
                    const chd64_evk *key);
int chd64_mult_const(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const uint64_t *cx,
                     double const_scale);
int chd64_add_const(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const uint64_t *cx);
int chd64_level_down(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, int target_level);

#ifdef __cplusplus
}
#endif

#endif /* CHEDDAR_B200_H_ */
