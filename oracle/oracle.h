/*
 * CPU oracle for the CKKS evaluation core — TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C11, the arithmetic of the reference
 * implementation (scale-snu/cheddar-fhe) on the hot path: signed Montgomery
 * arithmetic, prime/twiddle generation, the negacyclic NTT in bit-reversed
 * Montgomery form, base conversion (BConv) with centered inputs, ModUp /
 * ModDown / Rescale / merged ModDown+Rescale with the rational-rescale
 * restore constants, the key-switching inner product, automorphisms, and the
 * HMult / HRot / HConj / hoisted-rotation compositions.
 *
 * It is the checker for the CUDA path: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.  Nothing in the product links
 * or calls it.
 *
 * Data layout follows the reference: a polynomial is [num_primes][N] uint32
 * residues, prime order = terminal primes reversed, main primes, aux primes
 * (include/core/Parameter.h:198-206 of the reference).
 *
 * Parity status: the Montgomery primitives and prime utilities are pinned
 * against the reference's own sources (include/common/Basic.cuh and
 * include/common/PrimeUtils.h compiled from the reference tree, see
 * oracle/Makefile target `ref`).  The reference's NTT / ModSwitch kernels
 * cannot be compiled here (they need rmm and libtommath), so those parts are
 * pinned by definition (NTT = evaluation at psi^(2*brev(k)+1); BConv = the
 * CRT identity) and by the reference's own decryption-error criterion.
 */
#ifndef CHEDDAR_ORACLE_H_
#define CHEDDAR_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* ---- arithmetic primitives (restating include/common/Basic.cuh) ---- */
int32_t orc_mont_reduce_lazy(int64_t a, uint32_t q, int32_t q_inv);
int32_t orc_mont_mult_lazy(int32_t a, int32_t b, uint32_t q, int32_t q_inv);
uint32_t orc_mont_reduce(int64_t a, uint32_t q, int32_t q_inv);
uint32_t orc_mont_mult(uint32_t a, uint32_t b, uint32_t q, int32_t q_inv);
int32_t orc_normalize(uint32_t a, uint32_t q);

/* ---- prime utilities (restating include/common/PrimeUtils.h) ---- */
uint32_t orc_pow_mod(uint32_t a, int64_t e, uint32_t q);
uint32_t orc_inv_mod(uint32_t a, uint32_t q);
uint32_t orc_find_generator(uint32_t q);
uint32_t orc_primitive_root(int m, uint32_t q);
int32_t orc_inv_mod_base(uint32_t q);
uint32_t orc_to_mont(uint32_t a, uint32_t q);

/* ---- parameters / context ---- */
/* level_cfg: nlevels pairs (num_main, num_ter).  Returns NULL on invalid
 * parameters; orc_last_error() then describes the problem. */
orc_ctx *orc_create(int log_degree, double base_scale, int default_enc_level,
                    const int *level_cfg, int nlevels, const uint32_t *main_p,
                    int nmain, const uint32_t *aux_p, int naux,
                    const uint32_t *ter_p, int nter, int add_main, int add_ter);
void orc_destroy(orc_ctx *c);
const char *orc_last_error(void);
int orc_degree(const orc_ctx *c);
int orc_max_level(const orc_ctx *c);
int orc_alpha(const orc_ctx *c);
int orc_L(const orc_ctx *c);
int orc_max_ter(const orc_ctx *c);
/* (num_main, num_ter) of a level in [-1, max_level] */
int orc_level_np(const orc_ctx *c, int level, int *num_main, int *num_ter);
/* beta (number of ModUp digits) at a level, for the default aux count */
int orc_beta(const orc_ctx *c, int level);
/* Concatenated prime vector (ter reversed, main, aux) */
int orc_prime_vector(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                     uint32_t *out);
/* Global index (into ter-reversed ++ main ++ aux at max level) of each prime
 * in the np prime vector. */
int orc_prime_gidx(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                   int *out);
double orc_scale(const orc_ctx *c, int level);
double orc_rescale_prime_prod(const orc_ctx *c, int level);
int orc_galois_factor(const orc_ctx *c, int i);
/* Twiddle tables of a global prime index: psi_rev (Montgomery) and
 * psi_inv_rev (Montgomery), N words each. */
int orc_twiddles(const orc_ctx *c, int gidx, uint32_t *tw, uint32_t *itw);

/* ---- NTT (restating src/core/NTT.cu semantics) ---- */
/* In place over the limb set of np.  mont=1 multiplies by R on the way in
 * (NTT(..., montgomery_conversion=true)). */
int orc_ntt(const orc_ctx *c, int num_main, int num_ter, int num_aux,
            uint32_t *data, int mont);
/* INTT; mont=1 removes the Montgomery factor (default of the reference). */
int orc_intt(const orc_ctx *c, int num_main, int num_ter, int num_aux,
             uint32_t *data, int mont);
/* Single-limb transforms on a global prime index. */
int orc_ntt_limb(const orc_ctx *c, int gidx, uint32_t *limb, int mont);
int orc_intt_limb(const orc_ctx *c, int gidx, uint32_t *limb, int mont);

/* ---- base conversion ---- */
/* Exact: out[m][n] = (sum_k xt[k][n] * T[m][k]) * 2^-32 mod dst[m] */
int orc_bconv(const orc_ctx *c, const int32_t *xt, int K, const int32_t *table,
              const uint32_t *dst_primes, int M, uint32_t *out);
/* The reference's accumulation schedule (int64 partial sums renormalised
 * every 4 terms, then a lazy Montgomery reduction), for the equivalence
 * test against the exact form above.  Output is not forced canonical. */
int orc_bconv_ref_schedule(const orc_ctx *c, const int32_t *xt, int K,
                           const int32_t *table, const uint32_t *dst_primes,
                           int M, uint32_t *out);
/* BConv table T[m][k] = normalize((prod_{j!=k} src_j) * R^2 mod dst_m) */
int orc_bconv_table(const uint32_t *src, int K, const uint32_t *dst, int M,
                    int32_t *table);

/* ---- ModSwitch (restating src/core/ModSwitch.cu) ---- */
int orc_level_consts(const orc_ctx *c, int level, int kind, int digit,
                     uint32_t *c1, int32_t *table, uint32_t *inv,
                     uint32_t *pad, int *dims);
/* src: [num_q][N] (eval, Montgomery); dst: beta x [num_q + num_aux][N] */
int orc_modup(const orc_ctx *c, int level, const uint32_t *src, uint32_t *dst);
/* src [num_q + alpha][N] -> dst [num_q][N] */
int orc_moddown(const orc_ctx *c, int level, const uint32_t *src,
                uint32_t *dst);
/* src [num_q][N] -> dst [num_q(level-1)][N] */
int orc_rescale(const orc_ctx *c, int level, const uint32_t *src,
                uint32_t *dst);
/* src [num_q + alpha][N] -> dst [num_q(level-1)][N] */
int orc_moddown_rescale(const orc_ctx *c, int level, const uint32_t *src,
                        uint32_t *dst);

/* ---- element-wise (restating src/core/ElementWise.cu) ---- */
int orc_tensor(const orc_ctx *c, int num_main, int num_ter, const uint32_t *b1,
               const uint32_t *a1, const uint32_t *b2, const uint32_t *a2,
               uint32_t *d0, uint32_t *d1, uint32_t *d2);
/* dst = automorphism(src) for rotation amount r in [0, N/2] or -1 (conj) */
int orc_permute(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                int amount, const uint32_t *src, uint32_t *dst);
int orc_mult_imag_unit(const orc_ctx *c, int num_main, int num_ter,
                       const uint32_t *src, uint32_t *dst);

/* ---- evaluator (restating src/core/Context.cpp) ---- */
/* Evaluation keys are beta pairs over the max-level key basis
 * (all L q primes + alpha aux primes): key_bx/key_ax are beta x [L+alpha][N]. */
/* HMult: (b1,a1) x (b2,a2) at `level`, relinearise, optionally rescale. */
int orc_hmult(const orc_ctx *c, int level, const uint32_t *b1,
              const uint32_t *a1, const uint32_t *b2, const uint32_t *a2,
              const uint32_t *key_bx, const uint32_t *key_ax, int rescale,
              uint32_t *out_bx, uint32_t *out_ax);
/* MultKey then ModDown (key switch of a 2-part ciphertext) */
int orc_relinearize(const orc_ctx *c, int level, const uint32_t *d0,
                    const uint32_t *d1, const uint32_t *d2,
                    const uint32_t *key_bx, const uint32_t *key_ax, int rescale,
                    uint32_t *out_bx, uint32_t *out_ax);
int orc_mult_key(const orc_ctx *c, int level, const uint32_t *bx,
                 const uint32_t *ax, const uint32_t *key_bx,
                 const uint32_t *key_ax, uint32_t *out_bx, uint32_t *out_ax);
/* HRot = MultKey then Permute; amount in (0, N/2) */
int orc_hrot(const orc_ctx *c, int level, const uint32_t *bx,
             const uint32_t *ax, const uint32_t *key_bx,
             const uint32_t *key_ax, int amount, uint32_t *out_bx,
             uint32_t *out_ax);
int orc_hconj(const orc_ctx *c, int level, const uint32_t *bx,
              const uint32_t *ax, const uint32_t *key_bx,
              const uint32_t *key_ax, uint32_t *out_bx, uint32_t *out_ax);
/* Rescale of a ciphertext part list (n parts of [num_q][N]) */
int orc_rescale_ct(const orc_ctx *c, int level, int nparts, const uint32_t *src,
                   uint32_t *dst);
/* Hoisted baby-step rotations (restating Hoist.cu EvaluateBabyStep with the
 * fused key-mult): outputs stay in the extended basis Q u P, i.e. R outputs of
 * 2 x [num_q + alpha][N]. keys: R x (beta x [L+alpha][N]) for bx and ax. */
int orc_hoisted_rotate(const orc_ctx *c, int level, const uint32_t *bx,
                       const uint32_t *ax, int R, const int *amounts,
                       const uint32_t *const *key_bx,
                       const uint32_t *const *key_ax, uint32_t *out_bx,
                       uint32_t *out_ax);

/* ---- client side (test-only; restating src/UserInterface.cu) ---- */
/* Ternary secret of Hamming weight h over all L+alpha primes, NTT+Montgomery */
int orc_gen_secret(const orc_ctx *c, uint64_t seed, int h, uint32_t *s);
/* Evaluation key: encrypt target_s under enc_s over the max-level key basis.
 * Both secrets are [L+alpha][N] in NTT+Montgomery form. */
int orc_gen_evk(const orc_ctx *c, uint64_t seed, const uint32_t *enc_s,
                const uint32_t *target_s, uint32_t *key_bx, uint32_t *key_ax);
int orc_gen_mult_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                     uint32_t *key_bx, uint32_t *key_ax);
int orc_gen_rot_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                    int amount, uint32_t *key_bx, uint32_t *key_ax);
int orc_gen_conj_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                     uint32_t *key_bx, uint32_t *key_ax);
int orc_encrypt(const orc_ctx *c, uint64_t seed, const uint32_t *s, int level,
                const uint32_t *pt, uint32_t *bx, uint32_t *ax);
int orc_decrypt(const orc_ctx *c, const uint32_t *s, int level,
                const uint32_t *bx, const uint32_t *ax, uint32_t *pt);
/* Encode num_slots complex values at (level, scale, num_aux); pt is
 * [num_q + num_aux][N] in NTT+Montgomery form. */
int orc_encode(const orc_ctx *c, int level, double scale, const double *re,
               const double *im, int num_slots, int num_aux, uint32_t *pt);
int orc_decode(const orc_ctx *c, int level, double scale, const uint32_t *pt,
               int num_slots, double *re, double *im);
/* BootContext::ModUpToMax without sparse-secret encapsulation: level -1
 * (bx, ax) -> top level (res_bx, res_ax) */
int orc_modup_to_max(const orc_ctx *c, const uint32_t *bx, const uint32_t *ax,
                     uint32_t *res_bx, uint32_t *res_ax);
/* ... with sparse-secret encapsulation (DtS key at level -1, StD digit-0 key) */
int orc_modup_to_max_sse(const orc_ctx *c, const uint32_t *bx, const uint32_t *ax,
                         const uint32_t *dts_bx, const uint32_t *dts_ax,
                         const uint32_t *std_bx, const uint32_t *std_ax,
                         uint32_t *res_bx, uint32_t *res_ax);
/* EncodeConstant: one Montgomery word per prime */
int orc_encode_const(const orc_ctx *c, int level, double scale, double value,
                     int num_aux, uint32_t *cx);
/* Uniform residues for a global prime set (seeded), for synthetic inputs */
int orc_uniform(const orc_ctx *c, uint64_t seed, int num_main, int num_ter,
                int num_aux, uint32_t *out);

#ifdef __cplusplus
}
#endif

#endif /* CHEDDAR_ORACLE_H_ */
