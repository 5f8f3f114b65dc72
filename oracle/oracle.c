/*
 * CPU oracle for the CKKS evaluation core — TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the scope and the parity status.  Every function cites
 * the reference file:line whose semantics it restates.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef __int128 i128;

static __thread char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *orc_last_error(void) { return g_err; }

/* ========================================================================
 * Montgomery arithmetic, R = 2^32 — Basic.cuh:80-88 (__montgomery_reduction_
 * lazy<u32>), :120-125 (__mult_montgomery_lazy), :150-157 (ReduceMontgomery),
 * :251-260 (MultMontgomery), :229-239 (Normalize).
 * ====================================================================== */
int32_t orc_mont_reduce_lazy(int64_t a, uint32_t q, int32_t q_inv) {
  int32_t lo = (int32_t)(uint32_t)(uint64_t)a;
  int32_t hi = (int32_t)(a >> 32);
  int32_t t = (int32_t)((uint32_t)lo * (uint32_t)q_inv);
  int32_t th = (int32_t)(((int64_t)t * (int64_t)(int32_t)q) >> 32);
  return hi - th;
}
int32_t orc_mont_mult_lazy(int32_t a, int32_t b, uint32_t q, int32_t q_inv) {
  return orc_mont_reduce_lazy((int64_t)a * (int64_t)b, q, q_inv);
}
uint32_t orc_mont_reduce(int64_t a, uint32_t q, int32_t q_inv) {
  int32_t r = orc_mont_reduce_lazy(a, q, q_inv);
  if (r < 0) r += (int32_t)q;
  return (uint32_t)r;
}
uint32_t orc_mont_mult(uint32_t a, uint32_t b, uint32_t q, int32_t q_inv) {
  int32_t r = orc_mont_mult_lazy((int32_t)a, (int32_t)b, q, q_inv);
  if (r < 0) r += (int32_t)q;
  return (uint32_t)r;
}
int32_t orc_normalize(uint32_t a, uint32_t q) {
  int32_t r = (int32_t)a;
  if (a > (q >> 1)) r -= (int32_t)q;
  return r;
}
static inline uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) {
  uint32_t r = a + b;
  return r >= q ? r - q : r;
}
static inline uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t q) {
  int32_t r = (int32_t)a - (int32_t)b;
  return (uint32_t)(r < 0 ? r + (int32_t)q : r);
}
static inline uint32_t neg_mod(uint32_t a, uint32_t q) { return a ? q - a : 0; }

/* ========================================================================
 * Prime utilities — PrimeUtils.h:57-248
 * ====================================================================== */
static inline uint32_t mul_mod(uint32_t a, uint32_t b, uint32_t q) {
  return (uint32_t)(((uint64_t)a * b) % q);
}
static int64_t gcd_ext(int64_t a, int64_t b, int64_t *x, int64_t *y) {
  /* PrimeUtils.h:27-42 */
  if (a == 0) {
    *x = 0;
    *y = 1;
    return b;
  }
  int64_t x1, y1;
  int64_t g = gcd_ext(b % a, a, &x1, &y1);
  *x = y1 - (b / a) * x1;
  *y = x1;
  return g;
}
uint32_t orc_inv_mod(uint32_t a, uint32_t q) {
  /* PrimeUtils.h:71-83 */
  a %= q;
  if (a == 0) return 0;
  int64_t x, y;
  gcd_ext(a, q, &x, &y);
  if (x < 0) x += q;
  return (uint32_t)x;
}
uint32_t orc_pow_mod(uint32_t a, int64_t e, uint32_t q) {
  /* PrimeUtils.h:95-124 */
  a %= q;
  if (a == 0) return 0;
  uint32_t exp_mod = q - 1;
  e %= (int64_t)exp_mod;
  uint64_t v = (uint64_t)(e < 0 ? -e : e);
  int pos = (e >= 0);
  if (v > (exp_mod >> 1)) {
    v = exp_mod - v;
    pos = !pos;
  }
  if (!pos) a = orc_inv_mod(a, q);
  uint32_t r = 1;
  while (v) {
    if (v & 1) r = mul_mod(r, a, q);
    v >>= 1;
    a = mul_mod(a, a, q);
  }
  return r;
}
uint32_t orc_find_generator(uint32_t q) {
  /* PrimeUtils.h:135-170: smallest r >= 2 with r^(phi/f) != 1 for every
   * prime factor f of phi = q-1. */
  uint32_t phi = q - 1, t = phi;
  uint32_t f[32];
  int nf = 0;
  uint32_t sq = (uint32_t)sqrt((double)phi);
  for (uint32_t i = 2; i <= sq; i++) {
    if (t % i == 0) {
      f[nf++] = i;
      while (t % i == 0) t /= i;
      if (t == 1) break;
    }
  }
  if (t > 1) f[nf++] = t;
  for (uint32_t r = 2; r <= phi; r++) {
    int ok = 1;
    for (int k = 0; k < nf; k++)
      if (orc_pow_mod(r, (int64_t)(phi / f[k]), q) == 1) {
        ok = 0;
        break;
      }
    if (ok) return r;
  }
  return 0;
}
uint32_t orc_primitive_root(int m, uint32_t q) {
  /* PrimeUtils.h:180-196 */
  uint32_t g = orc_find_generator(q);
  if ((q - 1) % (uint32_t)m) return 0;
  return orc_pow_mod(g, (int64_t)((q - 1) / (uint32_t)m), q);
}
int32_t orc_inv_mod_base(uint32_t q) {
  /* PrimeUtils.h:205-231 computes q^-1 mod 2^32 as a signed word; the value
   * is unique in [-2^31, 2^31), so a Newton iteration gives the same word. */
  uint32_t x = q;
  for (int i = 0; i < 5; i++) x *= 2u - q * x;
  return (int32_t)x;
}
uint32_t orc_to_mont(uint32_t a, uint32_t q) {
  /* PrimeUtils.h:240-246 */
  return (uint32_t)(((uint64_t)a << 32) % q);
}
static unsigned brev(unsigned x, int bits) {
  unsigned r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

/* ========================================================================
 * Parameter / level model — Parameter.cu:20-194, 286-332
 * ====================================================================== */
typedef struct {
  int num_main, num_ter, num_aux;
} np_t;
static int np_q(np_t n) { return n.num_main + n.num_ter; }
static int np_total(np_t n) { return n.num_main + n.num_ter + n.num_aux; }

typedef struct {
  int level, num_aux, beta;
  int num_q;
  uint32_t *mod_up1;      /* [num_q] plain */
  int *dig_s, *dig_e;     /* relative digit ranges; dig_e <= 0 -> skipped */
  int32_t **mod_up2;      /* per digit [dst_len][src_len] */
  uint32_t *mod_down1;    /* [num_aux] */
  int32_t *mod_down2;     /* [num_q][num_aux] */
  uint32_t *inv_p_prod;   /* [num_q] Montgomery */
  int has_rescale;
  int pad_start, pad_end, restore_start, restore_end;
  int rs_src_len, mdr_src_len, rs_dst_len;
  uint32_t *rs1, *rs_inv, *rs_pad;
  int32_t *rs2;
  uint32_t *mdr1, *mdr_inv, *mdr_pad;
  int32_t *mdr2;
} msw_t;

struct orc_ctx {
  int log_n, n;
  int max_ter, max_main, L, alpha, dnum, max_level, nlevels;
  int (*lvl)[2];
  int add_main, add_ter;
  int def_enc_level;
  double base_scale;
  np_t short_np; /* level -1 base (num_aux = SSE aux count) */
  int nprimes;   /* L + alpha */
  uint32_t *primes;
  int32_t *qinv;
  uint32_t *tw, *itw; /* [nprimes][N] Montgomery psi_rev / psi_inv_rev */
  uint32_t *n_inv, *n_inv_mont, *mont_conv;
  uint32_t *p_prod; /* [L] Montgomery P mod q (all alpha aux) */
  int *galois;      /* [N/2 + 1] */
  double *scale, *rescale_prod;
  msw_t *msw; /* index level + 1, level in [-1, max_level] */
};

int orc_degree(const orc_ctx *c) { return c->n; }
int orc_max_level(const orc_ctx *c) { return c->max_level; }
int orc_alpha(const orc_ctx *c) { return c->alpha; }
int orc_L(const orc_ctx *c) { return c->L; }
int orc_max_ter(const orc_ctx *c) { return c->max_ter; }

static np_t level_np(const orc_ctx *c, int level, int num_aux) {
  /* Parameter.cu:286-296 */
  np_t r;
  if (level == -1) {
    r = c->short_np;
    r.num_aux = num_aux;
    return r;
  }
  r.num_main = c->lvl[level][0];
  r.num_ter = c->lvl[level][1];
  r.num_aux = num_aux;
  return r;
}
int orc_level_np(const orc_ctx *c, int level, int *num_main, int *num_ter) {
  if (level < -1 || level > c->max_level) {
    set_err("invalid level %d", level);
    return -1;
  }
  np_t n = level_np(c, level, 0);
  *num_main = n.num_main;
  *num_ter = n.num_ter;
  return 0;
}
/* Global index of each prime of np: ter reversed occupy [max_ter - t, max_ter),
 * main j is max_ter + j, aux a is L + a.  (Parameter.cu:317-325) */
static void np_gidx(const orc_ctx *c, np_t n, int *g) {
  int k = 0;
  for (int i = 0; i < n.num_ter + n.num_main; i++) g[k++] = c->max_ter - n.num_ter + i;
  for (int a = 0; a < n.num_aux; a++) g[k++] = c->L + a;
}
int orc_prime_gidx(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                   int *out) {
  np_t n = {num_main, num_ter, num_aux};
  np_gidx(c, n, out);
  return 0;
}
int orc_prime_vector(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                     uint32_t *out) {
  np_t n = {num_main, num_ter, num_aux};
  int g[256];
  np_gidx(c, n, g);
  for (int i = 0; i < np_total(n); i++) out[i] = c->primes[g[i]];
  return 0;
}
double orc_scale(const orc_ctx *c, int level) {
  if (level == -1) level = 0;
  if (level < 0 || level > c->def_enc_level) return 0.0;
  return c->scale[level];
}
double orc_rescale_prime_prod(const orc_ctx *c, int level) {
  if (level <= 0 || level > c->max_level) return 0.0;
  return c->rescale_prod[level];
}
int orc_galois_factor(const orc_ctx *c, int i) {
  if (i < 0 || i > c->n / 2) return -1;
  return c->galois[i];
}
int orc_twiddles(const orc_ctx *c, int g, uint32_t *tw, uint32_t *itw) {
  if (g < 0 || g >= c->nprimes) return -1;
  memcpy(tw, c->tw + (size_t)g * c->n, sizeof(uint32_t) * c->n);
  memcpy(itw, c->itw + (size_t)g * c->n, sizeof(uint32_t) * c->n);
  return 0;
}

/* ---- ModSwitch constants — ModSwitch.cu:320-370 and :372-411 ---- */
static void ms_consts(const orc_ctx *c, const uint32_t *src, int sl,
                      const uint32_t *dst, int dl, int rs, int re,
                      uint32_t *c1, int32_t *c2) {
  for (int i = 0; i < sl; i++) {
    uint32_t m = src[i], v = 1;
    for (int j = 0; j < sl; j++)
      if (j != i) v = mul_mod(v, src[j], m);
    v = mul_mod(v, (uint32_t)c->n, m);
    v = orc_inv_mod(v, m);
    for (int j = rs; j < re; j++) v = mul_mod(v, dst[j], m);
    c1[i] = v;
  }
  for (int mi = 0; mi < dl; mi++) {
    uint32_t p = dst[mi];
    for (int i = 0; i < sl; i++) {
      uint32_t acc = 1;
      for (int j = 0; j < sl; j++)
        if (j != i) acc = mul_mod(acc, src[j], p);
      acc = orc_to_mont(orc_to_mont(acc, p), p);
      c2[mi * sl + i] = orc_normalize(acc, p);
    }
  }
}
static void epi_consts(const uint32_t *src, int sl, const uint32_t *dst, int dl,
                       int rs, int re, uint32_t *inv, uint32_t *pad) {
  for (int i = 0; i < dl; i++) {
    uint32_t p = dst[i], v = 1;
    for (int j = 0; j < sl; j++) v = mul_mod(v, src[j], p);
    inv[i] = orc_to_mont(orc_inv_mod(v, p), p);
  }
  if (!pad) return;
  int rl = re - rs;
  for (int i = 0; i < dl - rl; i++) {
    int pi = i >= rs ? i + rl : i;
    uint32_t p = dst[pi], v = 1;
    for (int j = rs; j < re; j++) v = mul_mod(v, dst[j], p);
    pad[i] = orc_to_mont(v, p);
  }
}
int orc_bconv_table(const uint32_t *src, int K, const uint32_t *dst, int M,
                    int32_t *table) {
  for (int mi = 0; mi < M; mi++) {
    uint32_t p = dst[mi];
    for (int i = 0; i < K; i++) {
      uint32_t acc = 1;
      for (int j = 0; j < K; j++)
        if (j != i) acc = mul_mod(acc, src[j], p);
      acc = orc_to_mont(orc_to_mont(acc, p), p);
      table[mi * K + i] = orc_normalize(acc, p);
    }
  }
  return 0;
}

static int sse_num_aux(const orc_ctx *c) {
  /* Parameter.cu:260-264 */
  return c->lvl[0][0] + c->lvl[0][1] - c->add_main - c->add_ter;
}

static void msw_init(orc_ctx *c, msw_t *m, int level) {
  /* ModSwitch.cu:175-318 */
  memset(m, 0, sizeof *m);
  m->level = level;
  m->num_aux = level == -1 ? sse_num_aux(c) : c->alpha;
  np_t n = level_np(c, level, m->num_aux);
  int nq = np_q(n);
  m->num_q = nq;
  m->beta = level == -1 ? 1 : (n.num_main + c->max_ter + m->num_aux - 1) / m->num_aux;
  int tot = np_total(n);
  uint32_t lp[256];
  int g[256];
  np_gidx(c, n, g);
  for (int i = 0; i < tot; i++) lp[i] = c->primes[g[i]];
  int padded = (level == -1) ? nq : n.num_main + c->max_ter;
  int npad = padded - nq;
  m->mod_up1 = calloc(nq, sizeof(uint32_t));
  m->dig_s = calloc(m->beta, sizeof(int));
  m->dig_e = calloc(m->beta, sizeof(int));
  m->mod_up2 = calloc(m->beta, sizeof(int32_t *));
  for (int i = 0; i < m->beta; i++) {
    int s = i * m->num_aux, e = (i + 1) * m->num_aux;
    if (e > padded) e = padded;
    if (e <= npad) {
      m->dig_s[i] = 0;
      m->dig_e[i] = 0;
      continue;
    }
    s = s - npad < 0 ? 0 : s - npad;
    e = e - npad;
    m->dig_s[i] = s;
    m->dig_e[i] = e;
    int sl = e - s, dl = tot - sl;
    uint32_t dst[256];
    int k = 0;
    for (int j = 0; j < s; j++) dst[k++] = lp[j];
    for (int j = e; j < tot; j++) dst[k++] = lp[j];
    m->mod_up2[i] = calloc((size_t)dl * sl, sizeof(int32_t));
    ms_consts(c, lp + s, sl, dst, dl, 0, 0, m->mod_up1 + s, m->mod_up2[i]);
  }
  const uint32_t *qp = lp, *pp = lp + nq;
  m->mod_down1 = calloc(m->num_aux, sizeof(uint32_t));
  m->mod_down2 = calloc((size_t)nq * m->num_aux, sizeof(int32_t));
  m->inv_p_prod = calloc(nq, sizeof(uint32_t));
  ms_consts(c, pp, m->num_aux, qp, nq, 0, 0, m->mod_down1, m->mod_down2);
  epi_consts(pp, m->num_aux, qp, nq, 0, 0, m->inv_p_prod, NULL);
  if (level == -1 || level == 0) return;
  np_t nn = level_np(c, level - 1, m->num_aux);
  uint32_t np_[256];
  int gn[256];
  np_gidx(c, nn, gn);
  for (int i = 0; i < np_total(nn); i++) np_[i] = c->primes[gn[i]];
  int nnq = np_q(nn);
  int main_diff = n.num_main - nn.num_main, ter_diff = n.num_ter - nn.num_ter;
  uint32_t rs_src[256], mdr_src[256];
  int rsl = 0;
  if (ter_diff > 0) {
    for (int j = 0; j < ter_diff; j++) rs_src[rsl++] = lp[j];
    m->pad_start = 0;
    m->pad_end = nq - ter_diff;
    m->restore_start = nnq + main_diff;
    m->restore_end = nnq;
  } else if (main_diff > 0) {
    for (int j = nq - main_diff; j < nq; j++) rs_src[rsl++] = lp[j];
    m->pad_start = -ter_diff;
    m->pad_end = nq - main_diff - ter_diff;
    m->restore_start = 0;
    m->restore_end = -ter_diff;
  } else {
    return; /* invalid rescale amount: no rescale constants */
  }
  m->has_rescale = 1;
  memcpy(mdr_src, rs_src, rsl * sizeof(uint32_t));
  for (int j = 0; j < m->num_aux; j++) mdr_src[rsl + j] = pp[j];
  int mdl = rsl + m->num_aux;
  m->rs_src_len = rsl;
  m->mdr_src_len = mdl;
  m->rs_dst_len = nnq;
  int rl = m->restore_end - m->restore_start;
  m->rs1 = calloc(rsl, sizeof(uint32_t));
  m->rs2 = calloc((size_t)nnq * rsl, sizeof(int32_t));
  m->rs_inv = calloc(nnq, sizeof(uint32_t));
  m->rs_pad = calloc(nnq - rl + 1, sizeof(uint32_t));
  m->mdr1 = calloc(mdl, sizeof(uint32_t));
  m->mdr2 = calloc((size_t)nnq * mdl, sizeof(int32_t));
  m->mdr_inv = calloc(nnq, sizeof(uint32_t));
  m->mdr_pad = calloc(nnq - rl + 1, sizeof(uint32_t));
  ms_consts(c, rs_src, rsl, np_, nnq, m->restore_start, m->restore_end, m->rs1,
            m->rs2);
  epi_consts(rs_src, rsl, np_, nnq, m->restore_start, m->restore_end, m->rs_inv,
             m->rs_pad);
  ms_consts(c, mdr_src, mdl, np_, nnq, m->restore_start, m->restore_end,
            m->mdr1, m->mdr2);
  epi_consts(mdr_src, mdl, np_, nnq, m->restore_start, m->restore_end,
             m->mdr_inv, m->mdr_pad);
}
static void msw_free(msw_t *m) {
  free(m->mod_up1);
  for (int i = 0; i < m->beta; i++) free(m->mod_up2 ? m->mod_up2[i] : NULL);
  free(m->mod_up2);
  free(m->dig_s);
  free(m->dig_e);
  free(m->mod_down1);
  free(m->mod_down2);
  free(m->inv_p_prod);
  free(m->rs1);
  free(m->rs2);
  free(m->rs_inv);
  free(m->rs_pad);
  free(m->mdr1);
  free(m->mdr2);
  free(m->mdr_inv);
  free(m->mdr_pad);
}

static int cmp_pair(const int *a, const int *b) {
  /* Parameter.cu:10-15: a < b iff fewer total primes, or equal and fewer main */
  int at = a[0] + a[1], bt = b[0] + b[1];
  return (at < bt) || (at == bt && a[0] < b[0]);
}

orc_ctx *orc_create(int log_degree, double base_scale, int default_enc_level,
                    const int *level_cfg, int nlevels, const uint32_t *main_p,
                    int nmain, const uint32_t *aux_p, int naux,
                    const uint32_t *ter_p, int nter, int add_main, int add_ter) {
  /* Parameter.cu:20-194 checks and tables; NTT.cu:1233-1299 twiddles;
   * Context.cpp:78-103 p_prod. */
  if (log_degree < 12 || log_degree > 16) {
    set_err("log_degree must be in [12,16]");
    return NULL;
  }
  if (naux <= 0 || nmain <= 0 || nlevels <= 0 || nmain + nter + naux > 255) {
    set_err("invalid prime counts");
    return NULL;
  }
  int n = 1 << log_degree;
  uint32_t base = 2u * (uint32_t)n;
  const uint32_t *lists[3] = {main_p, aux_p, ter_p};
  int lens[3] = {nmain, naux, nter};
  for (int l = 0; l < 3; l++)
    for (int i = 0; i < lens[l]; i++) {
      if (lists[l][i] >= (1u << 31)) {
        set_err("Max prime is too large for the word size");
        return NULL;
      }
      if (lists[l][i] % base != 1) {
        set_err("Prime is not NTT-friendly");
        return NULL;
      }
    }
  int prev[2] = {0, 0};
  for (int i = 0; i < nlevels - 1; i++) {
    int cm = level_cfg[2 * i], ct = level_cfg[2 * i + 1];
    if (cm < 0 || cm > nmain || ct < 0 || ct > nter) {
      set_err("Invalid level configuration at level %d", i);
      return NULL;
    }
    if (!cmp_pair(prev, level_cfg + 2 * i)) {
      set_err("Invalid level configuration at level %d", i);
      return NULL;
    }
    prev[0] = cm;
    prev[1] = ct;
  }
  if (level_cfg[2 * (nlevels - 1)] != nmain ||
      level_cfg[2 * (nlevels - 1) + 1] != nter) {
    set_err("Invalid number of primes at the last level");
    return NULL;
  }
  orc_ctx *c = calloc(1, sizeof *c);
  c->log_n = log_degree;
  c->n = n;
  c->max_ter = nter;
  c->max_main = nmain;
  c->L = nmain + nter;
  c->alpha = naux;
  c->dnum = (c->L + naux - 1) / naux;
  c->nlevels = nlevels;
  c->max_level = nlevels - 1;
  c->lvl = calloc(nlevels, sizeof *c->lvl);
  for (int i = 0; i < nlevels; i++) {
    c->lvl[i][0] = level_cfg[2 * i];
    c->lvl[i][1] = level_cfg[2 * i + 1];
  }
  c->add_main = add_main;
  c->add_ter = add_ter;
  c->def_enc_level = default_enc_level;
  c->base_scale = base_scale;
  c->short_np.num_main = c->lvl[0][0] - add_main;
  c->short_np.num_ter = c->lvl[0][1] - add_ter;
  c->short_np.num_aux = c->short_np.num_main + c->short_np.num_ter;
  if (c->short_np.num_main < 0 || c->short_np.num_ter < 0 ||
      c->short_np.num_aux > naux) {
    set_err("Invalid additional base configuration");
    free(c->lvl);
    free(c);
    return NULL;
  }
  c->nprimes = c->L + naux;
  c->primes = calloc(c->nprimes, sizeof(uint32_t));
  for (int i = 0; i < nter; i++) c->primes[i] = ter_p[nter - 1 - i];
  for (int i = 0; i < nmain; i++) c->primes[nter + i] = main_p[i];
  for (int i = 0; i < naux; i++) c->primes[c->L + i] = aux_p[i];
  c->qinv = calloc(c->nprimes, sizeof(int32_t));
  c->n_inv = calloc(c->nprimes, sizeof(uint32_t));
  c->n_inv_mont = calloc(c->nprimes, sizeof(uint32_t));
  c->mont_conv = calloc(c->nprimes, sizeof(uint32_t));
  c->tw = malloc(sizeof(uint32_t) * (size_t)n * c->nprimes);
  c->itw = malloc(sizeof(uint32_t) * (size_t)n * c->nprimes);
#pragma omp parallel for schedule(dynamic)
  for (int g = 0; g < c->nprimes; g++) {
    uint32_t q = c->primes[g];
    c->qinv[g] = orc_inv_mod_base(q);
    uint32_t psi = orc_primitive_root(2 * n, q);
    uint32_t psi_inv = orc_inv_mod(psi, q);
    c->n_inv[g] = orc_inv_mod((uint32_t)n, q);
    c->n_inv_mont[g] = orc_to_mont(c->n_inv[g], q);
    c->mont_conv[g] = orc_to_mont(orc_to_mont(1, q), q);
    uint32_t *pw = malloc(sizeof(uint32_t) * n), *pwi = malloc(sizeof(uint32_t) * n);
    pw[0] = 1;
    pwi[0] = 1;
    for (int j = 1; j < n; j++) {
      pw[j] = mul_mod(pw[j - 1], psi, q);
      pwi[j] = mul_mod(pwi[j - 1], psi_inv, q);
    }
    for (int j = 0; j < n; j++) {
      unsigned r = brev((unsigned)j, log_degree);
      c->tw[(size_t)g * n + j] = orc_to_mont(pw[r], q);
      c->itw[(size_t)g * n + j] = orc_to_mont(pwi[r], q);
    }
    free(pw);
    free(pwi);
  }
  c->p_prod = calloc(c->L, sizeof(uint32_t));
  for (int i = 0; i < c->L; i++) {
    uint32_t q = c->primes[i], v = 1;
    for (int a = 0; a < naux; a++) v = mul_mod(v, c->primes[c->L + a], q);
    c->p_prod[i] = orc_to_mont(v, q);
  }
  c->galois = calloc(n / 2 + 1, sizeof(int));
  c->galois[0] = 1;
  c->galois[n / 2] = 1;
  for (int i = 1; i < n / 2; i++) c->galois[i] = (c->galois[i - 1] * 5) % (2 * n);
  c->rescale_prod = calloc(nlevels, sizeof(double));
  c->scale = calloc(default_enc_level + 1, sizeof(double));
  c->scale[0] = base_scale;
  double ns = base_scale;
  for (int i = 1; i <= c->max_level; i++) {
    np_t up = level_np(c, i, 0), lo = level_np(c, i - 1, 0);
    int td = up.num_ter - lo.num_ter, md = up.num_main - lo.num_main;
    double num = 1.0, den = 1.0;
    if (td >= 0)
      for (int j = 0; j < td; j++) num *= ter_p[lo.num_ter + j];
    else
      for (int j = 0; j < -td; j++) den *= ter_p[up.num_ter + j];
    if (md >= 0)
      for (int j = 0; j < md; j++) num *= main_p[lo.num_main + j];
    else
      for (int j = 0; j < -md; j++) den *= main_p[up.num_main + j];
    double prod = num / den;
    c->rescale_prod[i] = prod;
    if (i <= default_enc_level) {
      ns = sqrt(ns * prod);
      c->scale[i] = ns;
    }
  }
  c->msw = calloc(c->max_level + 2, sizeof(msw_t));
  for (int l = -1; l <= c->max_level; l++) msw_init(c, &c->msw[l + 1], l);
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  for (int l = -1; l <= c->max_level; l++) msw_free(&c->msw[l + 1]);
  free(c->msw);
  free(c->lvl);
  free(c->primes);
  free(c->qinv);
  free(c->n_inv);
  free(c->n_inv_mont);
  free(c->mont_conv);
  free(c->tw);
  free(c->itw);
  free(c->p_prod);
  free(c->galois);
  free(c->rescale_prod);
  free(c->scale);
  free(c);
}

int orc_beta(const orc_ctx *c, int level) {
  if (level < -1 || level > c->max_level) return -1;
  return c->msw[level + 1].beta;
}

/* ========================================================================
 * NTT — the reference's two-phase kernels (NTT.cu:231-454 forward,
 * NTT.cu:23-229 inverse) compute the standard negacyclic transform with the
 * bit-reversed Montgomery psi tables of NTT.cu:1258-1281.  The butterflies
 * below restate NTTUtils.cuh:19-60 (ButterflyNTT / ButterflyINTT) on signed
 * lazy values.
 * ====================================================================== */
static inline void bf_ntt(int32_t *a, int32_t *b, uint32_t w, uint32_t q,
                          int32_t qi) {
  int32_t x = *a;
  if (x < 0) x += (int32_t)q;
  int32_t m = orc_mont_mult_lazy(*b, (int32_t)w, q, qi);
  if (m < 0) m += (int32_t)q;
  *b = x - m;
  *a = (x - (int32_t)q) + m;
}
static inline void bf_intt(int32_t *a, int32_t *b, uint32_t w, uint32_t q,
                           int32_t qi) {
  int32_t x = *a, y = *b;
  if (x < 0) x += (int32_t)q;
  if (y < 0) y += (int32_t)q;
  int32_t d = x - y;
  *a = (x - (int32_t)q) + y;
  *b = orc_mont_mult_lazy(d, (int32_t)w, q, qi);
}
/* forward: optional pre-multiplication by a constant (MultConstLazy,
 * NTTUtils.cuh:361-368), stages with psi_rev[m + i], final canonicalisation. */
static void ntt_core(const orc_ctx *c, int g, int32_t *a, const uint32_t *pre) {
  int n = c->n;
  uint32_t q = c->primes[g];
  int32_t qi = c->qinv[g];
  const uint32_t *w = c->tw + (size_t)g * n;
  if (pre)
    for (int j = 0; j < n; j++) a[j] = orc_mont_mult_lazy(a[j], (int32_t)*pre, q, qi);
  for (int m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1)
    for (int i = 0; i < m; i++) {
      uint32_t wi = w[m + i];
      int32_t *x = a + 2 * i * t;
      for (int j = 0; j < t; j++) bf_ntt(x + j, x + j + t, wi, q, qi);
    }
  for (int j = 0; j < n; j++)
    if (a[j] < 0) a[j] += (int32_t)q;
}
/* inverse without the final constant; caller applies the epilogue */
static void intt_core(const orc_ctx *c, int g, int32_t *a) {
  int n = c->n;
  uint32_t q = c->primes[g];
  int32_t qi = c->qinv[g];
  const uint32_t *w = c->itw + (size_t)g * n;
  for (int m = n >> 1, t = 1; m >= 1; m >>= 1, t <<= 1)
    for (int i = 0; i < m; i++) {
      uint32_t wi = w[m + i];
      int32_t *x = a + 2 * i * t;
      for (int j = 0; j < t; j++) bf_intt(x + j, x + j + t, wi, q, qi);
    }
}
/* NTTUtils.cuh:370-391 MultConst / MultConstNormalize epilogues */
static inline int32_t ep_mult(int32_t v, uint32_t k, uint32_t q, int32_t qi) {
  int32_t t = orc_mont_mult_lazy(v, (int32_t)k, q, qi);
  if (t < 0) t += (int32_t)q;
  return t;
}
static inline int32_t ep_mult_norm(int32_t v, uint32_t k, uint32_t q, int32_t qi) {
  int32_t t = ep_mult(v, k, q, qi);
  if (t > (int32_t)(q >> 1)) t -= (int32_t)q;
  return t;
}

int orc_ntt_limb(const orc_ctx *c, int g, uint32_t *limb, int mont) {
  if (g < 0 || g >= c->nprimes) return -1;
  ntt_core(c, g, (int32_t *)limb, mont ? &c->mont_conv[g] : NULL);
  return 0;
}
int orc_intt_limb(const orc_ctx *c, int g, uint32_t *limb, int mont) {
  if (g < 0 || g >= c->nprimes) return -1;
  int32_t *a = (int32_t *)limb;
  intt_core(c, g, a);
  uint32_t k = mont ? c->n_inv[g] : c->n_inv_mont[g];
  for (int j = 0; j < c->n; j++) a[j] = ep_mult(a[j], k, c->primes[g], c->qinv[g]);
  return 0;
}
int orc_ntt(const orc_ctx *c, int num_main, int num_ter, int num_aux,
            uint32_t *data, int mont) {
  np_t n = {num_main, num_ter, num_aux};
  int g[256];
  np_gidx(c, n, g);
  int tot = np_total(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < tot; i++) orc_ntt_limb(c, g[i], data + (size_t)i * c->n, mont);
  return 0;
}
int orc_intt(const orc_ctx *c, int num_main, int num_ter, int num_aux,
             uint32_t *data, int mont) {
  np_t n = {num_main, num_ter, num_aux};
  int g[256];
  np_gidx(c, n, g);
  int tot = np_total(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < tot; i++) orc_intt_limb(c, g[i], data + (size_t)i * c->n, mont);
  return 0;
}

/* ========================================================================
 * BConv — ModSwitch.cu:23-171 (ModSwitchMatrixMult).  The output residue is
 * (sum_k xt_k * T_mk) * R^-1 mod p_m; computed exactly here.
 * ====================================================================== */
static void bconv_exact(const int32_t *xt, int K, const int32_t *T,
                        const uint32_t *dst, const int32_t *dqinv, int M,
                        int n, uint32_t *const *out_rows) {
#pragma omp parallel for schedule(static)
  for (int m = 0; m < M; m++) {
    uint32_t p = dst[m];
    int32_t pinv = dqinv[m];
    uint32_t *o = out_rows[m];
    for (int j = 0; j < n; j++) {
      i128 acc = 0;
      for (int k = 0; k < K; k++) acc += (int64_t)xt[(size_t)k * n + j] * T[m * K + k];
      int64_t r = (int64_t)(acc % (i128)p);
      if (r < 0) r += p;
      o[j] = orc_mont_reduce(r, p, pinv);
    }
  }
}
int orc_bconv(const orc_ctx *c, const int32_t *xt, int K, const int32_t *table,
              const uint32_t *dst_primes, int M, uint32_t *out) {
  int32_t qi[256];
  uint32_t *rows[256];
  for (int m = 0; m < M; m++) {
    qi[m] = orc_inv_mod_base(dst_primes[m]);
    rows[m] = out + (size_t)m * c->n;
  }
  bconv_exact(xt, K, table, dst_primes, qi, M, c->n, rows);
  return 0;
}
int orc_bconv_ref_schedule(const orc_ctx *c, const int32_t *xt, int K,
                           const int32_t *table, const uint32_t *dst_primes,
                           int M, uint32_t *out) {
  /* ModSwitch.cu:98-170 accumulation order: groups of 4 source limbs, an
   * int64 renormalisation into [-p*2^31, p*2^31) after each full group,
   * then ReduceMontgomery. */
  int n = c->n;
  for (int m = 0; m < M; m++) {
    uint32_t p = dst_primes[m];
    int32_t pinv = orc_inv_mod_base(p);
    int64_t th = (int64_t)p << 32, half = th >> 1;
    for (int j = 0; j < n; j++) {
      int64_t acc = 0;
      int cnt = 0;
      for (int i = 0; i < K; i += 4) {
        for (int k = i; k < i + 4 && k < K; k++) {
          acc += (int64_t)xt[(size_t)k * n + j] * (int64_t)table[m * K + k];
          cnt++;
        }
        if (cnt >= 4) {
          if (acc < 0) acc += th;
          if (acc >= half) acc -= th;
          cnt -= 4;
        }
      }
      out[(size_t)m * n + j] = orc_mont_reduce(acc, p, pinv);
    }
  }
  return 0;
}

/* ========================================================================
 * ModUp — ModSwitch.cu:429-509
 * ====================================================================== */
static int modup_impl(const orc_ctx *c, const msw_t *m, np_t n,
                      const uint32_t *src, uint32_t *dst) {
  int N = c->n, nq = np_q(n), na = m->num_aux, tot = nq + na;
  n.num_aux = na;
  int g[256];
  np_gidx(c, n, g);
  /* INTTAndMultConst(normalize=true) with mod_up1: centered x~ */
  int32_t *xt = malloc(sizeof(int32_t) * (size_t)nq * N);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nq; i++) {
    int32_t *a = xt + (size_t)i * N;
    memcpy(a, src + (size_t)i * N, sizeof(int32_t) * N);
    intt_core(c, g[i], a);
    for (int j = 0; j < N; j++)
      a[j] = ep_mult_norm(a[j], m->mod_up1[i], c->primes[g[i]], c->qinv[g[i]]);
  }
  for (int d = 0; d < m->beta; d++) {
    int s = m->dig_s[d], e = m->dig_e[d];
    uint32_t *out = dst + (size_t)d * tot * N;
    if (e <= 0) continue;
    int sl = e - s;
    memcpy(out + (size_t)s * N, src + (size_t)s * N, sizeof(uint32_t) * sl * N);
    uint32_t dp[256];
    int32_t dqi[256];
    uint32_t *rows[256];
    int k = 0;
    for (int j = 0; j < tot; j++) {
      if (j >= s && j < e) continue;
      dp[k] = c->primes[g[j]];
      dqi[k] = c->qinv[g[j]];
      rows[k] = out + (size_t)j * N;
      k++;
    }
    bconv_exact(xt + (size_t)s * N, sl, m->mod_up2[d], dp, dqi, k, N, rows);
    /* NTTForModUp (no Montgomery conversion), skipping the digit's primes */
#pragma omp parallel for schedule(static)
    for (int j = 0; j < tot; j++) {
      if (j >= s && j < e) continue;
      ntt_core(c, g[j], (int32_t *)(out + (size_t)j * N), NULL);
    }
  }
  free(xt);
  return 0;
}
int orc_modup(const orc_ctx *c, int level, const uint32_t *src, uint32_t *dst) {
  if (level < -1 || level > c->max_level) return -1;
  const msw_t *m = &c->msw[level + 1];
  return modup_impl(c, m, level_np(c, level, 0), src, dst);
}

/* ========================================================================
 * ModDown / Rescale / ModDownAndRescale — ModSwitch.cu:511-684 with
 * NTT.cu:973-1128 (INTTForModDown) and NTT.cu:456-601 + :889-971
 * (NTTForModDown epilogue (src2 * pad - x) * inv_prod).
 * ====================================================================== */
enum { MD_MODDOWN = 0, MD_RESCALE = 1, MD_MDR = 2 };
static int moddown_worker(const orc_ctx *c, int level, int type,
                          const uint32_t *src, uint32_t *dst) {
  const msw_t *m = &c->msw[level + 1];
  int N = c->n;
  int nsa = type == MD_RESCALE ? 0 : m->num_aux;
  np_t ns = level_np(c, level, nsa);
  np_t nd = level_np(c, type == MD_MODDOWN ? level : level - 1, 0);
  np_t nn = {ns.num_main < nd.num_main ? ns.num_main : nd.num_main,
             ns.num_ter < nd.num_ter ? ns.num_ter : nd.num_ter, 0};
  int src_len = np_total(ns) - np_total(nn);
  int dst_len = np_total(nd);
  if (type != MD_MODDOWN && !m->has_rescale) {
    set_err("no rescale at level %d", level);
    return -1;
  }
  const uint32_t *c1 = type == MD_MODDOWN ? m->mod_down1 : type == MD_RESCALE ? m->rs1 : m->mdr1;
  const int32_t *c2 = type == MD_MODDOWN ? m->mod_down2 : type == MD_RESCALE ? m->rs2 : m->mdr2;
  const uint32_t *inv = type == MD_MODDOWN ? m->inv_p_prod : type == MD_RESCALE ? m->rs_inv : m->mdr_inv;
  const uint32_t *pad = type == MD_MODDOWN ? NULL : type == MD_RESCALE ? m->rs_pad : m->mdr_pad;
  int gs[256];
  np_gidx(c, ns, gs);
  /* rows of src that are INTT'd: dropped q primes then aux */
  int rows[256], nr = 0;
  int on_main = ns.num_main > nn.num_main, on_ter = ns.num_ter > nn.num_ter;
  if (on_main && on_ter) {
    set_err("INTTForModDown: invalid np combination");
    return -1;
  }
  if (!on_ter) {
    for (int r = ns.num_ter + nn.num_main; r < np_q(ns); r++) rows[nr++] = r;
  } else {
    for (int r = 0; r < ns.num_ter - nn.num_ter; r++) rows[nr++] = r;
  }
  for (int a = 0; a < nsa; a++) rows[nr++] = np_q(ns) + a;
  if (nr != src_len) {
    set_err("internal: src_len mismatch");
    return -1;
  }
  int32_t *xt = malloc(sizeof(int32_t) * (size_t)src_len * N);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < src_len; i++) {
    int g = gs[rows[i]];
    int32_t *a = xt + (size_t)i * N;
    memcpy(a, src + (size_t)rows[i] * N, sizeof(int32_t) * N);
    intt_core(c, g, a);
    for (int j = 0; j < N; j++) a[j] = ep_mult_norm(a[j], c1[i], c->primes[g], c->qinv[g]);
  }
  int gd[256];
  np_gidx(c, nd, gd);
  uint32_t dp[256];
  int32_t dqi[256];
  uint32_t *orow[256];
  for (int y = 0; y < dst_len; y++) {
    dp[y] = c->primes[gd[y]];
    dqi[y] = c->qinv[gd[y]];
    orow[y] = dst + (size_t)y * N;
  }
  bconv_exact(xt, src_len, c2, dp, dqi, dst_len, N, orow);
  free(xt);
  int src2_start = nd.num_ter - nn.num_ter;
  int src2_end = src2_start + np_q(nn);
  int src2_off = ns.num_ter - nd.num_ter;
  if (src2_off < 0) src2_off = 0;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < dst_len; y++) {
    int32_t *o = (int32_t *)orow[y];
    ntt_core(c, gd[y], o, NULL);
    uint32_t q = dp[y];
    int32_t qi = dqi[y];
    int exists = (y >= src2_start && y < src2_end);
    const uint32_t *s2 = exists ? src + (size_t)(src2_off + y - src2_start) * N : NULL;
    int32_t padv = (exists && pad) ? (int32_t)pad[y - src2_start] : 0;
    for (int j = 0; j < N; j++) {
      int32_t r = 0;
      if (exists) {
        r = (int32_t)s2[j];
        if (pad) {
          r = orc_mont_mult_lazy(r, padv, q, qi);
          if (r < 0) r += (int32_t)q;
        }
      }
      r -= o[j];
      r = orc_mont_mult_lazy(r, (int32_t)inv[y], q, qi);
      if (r < 0) r += (int32_t)q;
      o[j] = r;
    }
  }
  return 0;
}
int orc_moddown(const orc_ctx *c, int level, const uint32_t *src, uint32_t *dst) {
  if (level < -1 || level > c->max_level) return -1;
  return moddown_worker(c, level, MD_MODDOWN, src, dst);
}
int orc_rescale(const orc_ctx *c, int level, const uint32_t *src, uint32_t *dst) {
  if (level < 1 || level > c->max_level) return -1;
  return moddown_worker(c, level, MD_RESCALE, src, dst);
}
int orc_moddown_rescale(const orc_ctx *c, int level, const uint32_t *src,
                        uint32_t *dst) {
  if (level < 1 || level > c->max_level) return -1;
  return moddown_worker(c, level, MD_MDR, src, dst);
}

/* ========================================================================
 * Element-wise — ElementWise.cu:504-575 (Tensor), :370-391 (Permute),
 * :625-658 (MultImaginaryUnit), :225-366 (CPAccum)
 * ====================================================================== */
int orc_tensor(const orc_ctx *c, int num_main, int num_ter, const uint32_t *b1,
               const uint32_t *a1, const uint32_t *b2, const uint32_t *a2,
               uint32_t *d0, uint32_t *d1, uint32_t *d2) {
  np_t n = {num_main, num_ter, 0};
  int g[256];
  np_gidx(c, n, g);
  int N = c->n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np_q(n); i++) {
    uint32_t q = c->primes[g[i]];
    int32_t qi = c->qinv[g[i]];
    for (int j = 0; j < N; j++) {
      size_t k = (size_t)i * N + j;
      uint32_t x0 = orc_mont_mult(b1[k], b2[k], q, qi);
      uint32_t x2 = orc_mont_mult(a1[k], a2[k], q, qi);
      int32_t s1 = ((int32_t)b1[k] - (int32_t)q) + (int32_t)a1[k];
      int32_t s2 = ((int32_t)b2[k] - (int32_t)q) + (int32_t)a2[k];
      uint32_t x1 = orc_mont_reduce((int64_t)s1 * s2, q, qi);
      x1 = sub_mod(x1, x0, q);
      x1 = sub_mod(x1, x2, q);
      d0[k] = x0;
      d1[k] = x1;
      d2[k] = x2;
    }
  }
  return 0;
}
static uint32_t galois_of(const orc_ctx *c, int amount) {
  /* ElementWise.cu:955-964 */
  if (amount == -1) return 2u * c->n - 1;
  return (uint32_t)c->galois[amount];
}
static void permute_rows(const orc_ctx *c, int nrows, uint32_t gf,
                         const uint32_t *src, uint32_t *dst) {
  /* ElementWise.cu:370-391: dst[k] = src[brev(brev(k)*2+1)*gf - 1)] */
  int N = c->n, lb = c->log_n + 1;
  uint32_t mask = (1u << lb) - 1;
  int *map = malloc(sizeof(int) * N);
  for (int k = 0; k < N; k++) {
    uint32_t xr = brev((unsigned)k, lb) + 1;
    uint32_t t = (xr * gf - 1) & mask;
    map[k] = (int)brev(t, lb);
  }
#pragma omp parallel for schedule(static)
  for (int r = 0; r < nrows; r++)
    for (int k = 0; k < N; k++) dst[(size_t)r * N + k] = src[(size_t)r * N + map[k]];
  free(map);
}
int orc_permute(const orc_ctx *c, int num_main, int num_ter, int num_aux,
                int amount, const uint32_t *src, uint32_t *dst) {
  if (!(amount == -1 || (amount >= 0 && amount <= c->n / 2))) return -1;
  np_t n = {num_main, num_ter, num_aux};
  permute_rows(c, np_total(n), galois_of(c, amount), src, dst);
  return 0;
}
int orc_mult_imag_unit(const orc_ctx *c, int num_main, int num_ter,
                       const uint32_t *src, uint32_t *dst) {
  np_t n = {num_main, num_ter, 0};
  int g[256];
  np_gidx(c, n, g);
  int N = c->n;
  for (int i = 0; i < np_q(n); i++) {
    uint32_t q = c->primes[g[i]];
    int32_t qi = c->qinv[g[i]];
    uint32_t u = c->tw[(size_t)g[i] * N + 1];
    for (int j = 0; j < N; j++) {
      uint32_t v = (j & (N / 2)) ? q - u : u;
      dst[(size_t)i * N + j] = orc_mont_mult(src[(size_t)i * N + j], v, q, qi);
    }
  }
  return 0;
}

/* ========================================================================
 * Key switching — Context.cpp:609-712 (MultKeyNoModDown), :584-607 (MultKey),
 * :714-737 (RelinearizeRescale), :776-791 (HRot), :862-871 (HMult)
 * ====================================================================== */
/* accum (2 x [nq+alpha][N]) = sum_i modup_i (.) key_i, then
 * accum_bx[q] += P * d0 and (if d1) accum_ax[q] += P * d1.  d_in is the
 * polynomial that is ModUp'ed. */
static int mult_key_no_moddown(const orc_ctx *c, int level, const uint32_t *d0,
                               const uint32_t *d1, const uint32_t *d_in,
                               const uint32_t *key_bx, const uint32_t *key_ax,
                               uint32_t *acc_bx, uint32_t *acc_ax) {
  const msw_t *m = &c->msw[level + 1];
  np_t n = level_np(c, level, c->alpha);
  int N = c->n, nq = np_q(n), na = c->alpha, tot = nq + na;
  int prime_offset = c->max_ter - n.num_ter;
  size_t dsz = (size_t)tot * N;
  uint32_t *mu = calloc((size_t)m->beta * dsz, sizeof(uint32_t));
  if (modup_impl(c, m, level_np(c, level, 0), d_in, mu)) return -1;
  int g[256];
  np_gidx(c, n, g);
  size_t ksz = (size_t)(c->L + na) * N;
#pragma omp parallel for schedule(static)
  for (int r = 0; r < tot; r++) {
    uint32_t q = c->primes[g[r]];
    int32_t qi = c->qinv[g[r]];
    int krow = r < nq ? prime_offset + r : c->L + (r - nq);
    for (int j = 0; j < N; j++) {
      uint32_t sb = 0, sa = 0;
      for (int d = 0; d < m->beta; d++) {
        if (m->dig_e[d] <= 0) continue;
        uint32_t v = mu[(size_t)d * dsz + (size_t)r * N + j];
        const uint32_t *kb = key_bx + (size_t)d * ksz + (size_t)krow * N;
        const uint32_t *ka = key_ax + (size_t)d * ksz + (size_t)krow * N;
        sb = add_mod(sb, orc_mont_mult(kb[j], v, q, qi), q);
        sa = add_mod(sa, orc_mont_mult(ka[j], v, q, qi), q);
      }
      if (r < nq) {
        uint32_t pp = c->p_prod[prime_offset + r];
        sb = add_mod(sb, orc_mont_mult(pp, d0[(size_t)r * N + j], q, qi), q);
        if (d1) sa = add_mod(sa, orc_mont_mult(pp, d1[(size_t)r * N + j], q, qi), q);
      }
      acc_bx[(size_t)r * N + j] = sb;
      acc_ax[(size_t)r * N + j] = sa;
    }
  }
  free(mu);
  return 0;
}

int orc_hmult(const orc_ctx *c, int level, const uint32_t *b1,
              const uint32_t *a1, const uint32_t *b2, const uint32_t *a2,
              const uint32_t *key_bx, const uint32_t *key_ax, int rescale,
              uint32_t *out_bx, uint32_t *out_ax) {
  if (level < 0 || level > c->max_level || (rescale && level < 1)) {
    set_err("invalid level");
    return -1;
  }
  np_t n = level_np(c, level, 0);
  int N = c->n, nq = np_q(n), tot = nq + c->alpha;
  size_t qs = (size_t)nq * N;
  uint32_t *d = malloc(3 * qs * sizeof(uint32_t));
  orc_tensor(c, n.num_main, n.num_ter, b1, a1, b2, a2, d, d + qs, d + 2 * qs);
  uint32_t *acc = malloc(2 * (size_t)tot * N * sizeof(uint32_t));
  uint32_t *ab = acc, *aa = acc + (size_t)tot * N;
  int rc = mult_key_no_moddown(c, level, d, d + qs, d + 2 * qs, key_bx, key_ax, ab, aa);
  if (!rc) {
    if (rescale) {
      rc = moddown_worker(c, level, MD_MDR, ab, out_bx);
      if (!rc) rc = moddown_worker(c, level, MD_MDR, aa, out_ax);
    } else {
      rc = moddown_worker(c, level, MD_MODDOWN, ab, out_bx);
      if (!rc) rc = moddown_worker(c, level, MD_MODDOWN, aa, out_ax);
    }
  }
  free(acc);
  free(d);
  return rc;
}

/* Context::Relinearize / RelinearizeRescale (Context.cpp:539-547, 714-737)
 * of a three-part ciphertext (d0, d1, d2) */
int orc_relinearize(const orc_ctx *c, int level, const uint32_t *d0,
                    const uint32_t *d1, const uint32_t *d2,
                    const uint32_t *key_bx, const uint32_t *key_ax, int rescale,
                    uint32_t *out_bx, uint32_t *out_ax) {
  if (level < 0 || level > c->max_level || (rescale && level < 1)) {
    set_err("invalid level");
    return -1;
  }
  np_t n = level_np(c, level, 0);
  int N = c->n, tot = np_q(n) + c->alpha;
  uint32_t *acc = malloc(2 * (size_t)tot * N * sizeof(uint32_t));
  uint32_t *ab = acc, *aa = acc + (size_t)tot * N;
  int rc = mult_key_no_moddown(c, level, d0, d1, d2, key_bx, key_ax, ab, aa);
  int md = rescale ? MD_MDR : MD_MODDOWN;
  if (!rc) rc = moddown_worker(c, level, md, ab, out_bx);
  if (!rc) rc = moddown_worker(c, level, md, aa, out_ax);
  free(acc);
  return rc;
}

int orc_mult_key(const orc_ctx *c, int level, const uint32_t *bx,
                 const uint32_t *ax, const uint32_t *key_bx,
                 const uint32_t *key_ax, uint32_t *out_bx, uint32_t *out_ax) {
  if (level < 0 || level > c->max_level) return -1;
  np_t n = level_np(c, level, 0);
  int N = c->n, tot = np_q(n) + c->alpha;
  uint32_t *acc = malloc(2 * (size_t)tot * N * sizeof(uint32_t));
  uint32_t *ab = acc, *aa = acc + (size_t)tot * N;
  int rc = mult_key_no_moddown(c, level, bx, NULL, ax, key_bx, key_ax, ab, aa);
  if (!rc) rc = moddown_worker(c, level, MD_MODDOWN, ab, out_bx);
  if (!rc) rc = moddown_worker(c, level, MD_MODDOWN, aa, out_ax);
  free(acc);
  return rc;
}

int orc_hrot(const orc_ctx *c, int level, const uint32_t *bx,
             const uint32_t *ax, const uint32_t *key_bx,
             const uint32_t *key_ax, int amount, uint32_t *out_bx,
             uint32_t *out_ax) {
  if (amount <= 0 || amount >= c->n / 2) return -1;
  np_t n = level_np(c, level, 0);
  size_t qs = (size_t)np_q(n) * c->n;
  uint32_t *t = malloc(2 * qs * sizeof(uint32_t));
  int rc = orc_mult_key(c, level, bx, ax, key_bx, key_ax, t, t + qs);
  if (!rc) {
    permute_rows(c, np_q(n), galois_of(c, amount), t, out_bx);
    permute_rows(c, np_q(n), galois_of(c, amount), t + qs, out_ax);
  }
  free(t);
  return rc;
}
int orc_hconj(const orc_ctx *c, int level, const uint32_t *bx,
              const uint32_t *ax, const uint32_t *key_bx,
              const uint32_t *key_ax, uint32_t *out_bx, uint32_t *out_ax) {
  np_t n = level_np(c, level, 0);
  size_t qs = (size_t)np_q(n) * c->n;
  uint32_t *t = malloc(2 * qs * sizeof(uint32_t));
  int rc = orc_mult_key(c, level, bx, ax, key_bx, key_ax, t, t + qs);
  if (!rc) {
    permute_rows(c, np_q(n), galois_of(c, -1), t, out_bx);
    permute_rows(c, np_q(n), galois_of(c, -1), t + qs, out_ax);
  }
  free(t);
  return rc;
}
int orc_rescale_ct(const orc_ctx *c, int level, int nparts, const uint32_t *src,
                   uint32_t *dst) {
  np_t n = level_np(c, level, 0), nn = level_np(c, level - 1, 0);
  size_t qs = (size_t)np_q(n) * c->n, qd = (size_t)np_q(nn) * c->n;
  for (int p = 0; p < nparts; p++) {
    int rc = moddown_worker(c, level, MD_RESCALE, src + p * qs, dst + p * qd);
    if (rc) return rc;
  }
  return 0;
}

int orc_hoisted_rotate(const orc_ctx *c, int level, const uint32_t *bx,
                       const uint32_t *ax, int R, const int *amounts,
                       const uint32_t *const *key_bx,
                       const uint32_t *const *key_ax, uint32_t *out_bx,
                       uint32_t *out_ax) {
  /* Hoist.cu:578-691 + BSFusedKernel (Hoist.cu:21-78): ModUp(ax) once; per
   * rotation sum_i modup_i (.) key_i (+ P*bx on q primes), then the
   * automorphism for the rotation amount, all in the Q u P basis. */
  if (level < 0 || level > c->max_level) return -1;
  const msw_t *m = &c->msw[level + 1];
  np_t n = level_np(c, level, c->alpha);
  int N = c->n, nq = np_q(n), na = c->alpha, tot = nq + na;
  int prime_offset = c->max_ter - n.num_ter;
  size_t dsz = (size_t)tot * N, ksz = (size_t)(c->L + na) * N;
  uint32_t *mu = calloc((size_t)m->beta * dsz, sizeof(uint32_t));
  modup_impl(c, m, level_np(c, level, 0), ax, mu);
  int g[256];
  np_gidx(c, n, g);
  uint32_t *tb = malloc(dsz * sizeof(uint32_t)), *ta = malloc(dsz * sizeof(uint32_t));
  for (int k = 0; k < R; k++) {
    if (amounts[k] <= 0 || amounts[k] >= N / 2) {
      free(mu);
      free(tb);
      free(ta);
      return -1;
    }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < tot; r++) {
      uint32_t q = c->primes[g[r]];
      int32_t qi = c->qinv[g[r]];
      int krow = r < nq ? prime_offset + r : c->L + (r - nq);
      for (int j = 0; j < N; j++) {
        uint32_t sb = 0, sa = 0;
        for (int d = 0; d < m->beta; d++) {
          if (m->dig_e[d] <= 0) continue;
          uint32_t v = mu[(size_t)d * dsz + (size_t)r * N + j];
          sb = add_mod(sb, orc_mont_mult(v, key_bx[k][(size_t)d * ksz + (size_t)krow * N + j], q, qi), q);
          sa = add_mod(sa, orc_mont_mult(v, key_ax[k][(size_t)d * ksz + (size_t)krow * N + j], q, qi), q);
        }
        if (r < nq)
          sb = add_mod(sb, orc_mont_mult(bx[(size_t)r * N + j], c->p_prod[prime_offset + r], q, qi), q);
        tb[(size_t)r * N + j] = sb;
        ta[(size_t)r * N + j] = sa;
      }
    }
    permute_rows(c, tot, galois_of(c, amounts[k]), tb, out_bx + (size_t)k * dsz);
    permute_rows(c, tot, galois_of(c, amounts[k]), ta, out_ax + (size_t)k * dsz);
  }
  free(tb);
  free(ta);
  free(mu);
  return 0;
}

/* ========================================================================
 * Client side (test-only) — UserInterface.cu:224-458, Random.h
 * A seeded xoshiro256** generator stands in for the reference's unseeded
 * mt19937_64; the distributions are the reference's.
 * ====================================================================== */
typedef struct {
  uint64_t s[4];
} rng_t;
static uint64_t splitmix(uint64_t *x) {
  uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed) {
  for (int i = 0; i < 4; i++) r->s[i] = splitmix(&seed);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t *r) {
  uint64_t *s = r->s;
  uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return res;
}
static uint64_t rng_below(rng_t *r, uint64_t bound) {
  /* unbiased uniform in [0, bound) */
  uint64_t lim = UINT64_MAX - UINT64_MAX % bound;
  uint64_t x;
  do x = rng_next(r);
  while (x >= lim);
  return x % bound;
}
static double rng_unit(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

int orc_uniform(const orc_ctx *c, uint64_t seed, int num_main, int num_ter,
                int num_aux, uint32_t *out) {
  np_t n = {num_main, num_ter, num_aux};
  int g[256];
  np_gidx(c, n, g);
  rng_t r;
  rng_seed(&r, seed);
  for (int i = 0; i < np_total(n); i++)
    for (int j = 0; j < c->n; j++) out[(size_t)i * c->n + j] = (uint32_t)rng_below(&r, c->primes[g[i]]);
  return 0;
}

int orc_gen_secret(const orc_ctx *c, uint64_t seed, int h, uint32_t *s) {
  /* UserInterface.cu:224-276: h distinct positions, values +-1 */
  int N = c->n;
  if (h < 1 || h > N) return -1;
  rng_t r;
  rng_seed(&r, seed);
  int *idx = malloc(sizeof(int) * N);
  for (int i = 0; i < N; i++) idx[i] = i;
  for (int i = 0; i < h; i++) {
    int j = i + (int)rng_below(&r, (uint64_t)(N - i));
    int t = idx[i];
    idx[i] = idx[j];
    idx[j] = t;
  }
  int *val = malloc(sizeof(int) * h);
  for (int i = 0; i < h; i++) val[i] = (int)rng_below(&r, 2);
  memset(s, 0, sizeof(uint32_t) * (size_t)c->nprimes * N);
  for (int g = 0; g < c->nprimes; g++) {
    uint32_t p = c->primes[g];
    for (int i = 0; i < h; i++) s[(size_t)g * N + idx[i]] = (p - 2) * (uint32_t)val[i] + 1;
  }
  free(idx);
  free(val);
  for (int g = 0; g < c->nprimes; g++) orc_ntt_limb(c, g, s + (size_t)g * N, 1);
  return 0;
}

/* Gaussian error (Random.h:62-75: sigma 3.2, clamp 6 sigma, llround) over the
 * rows of gidx g[0..nrows), NTT+Montgomery (UserInterface.cu:488-520) */
static void sample_error(const orc_ctx *c, rng_t *r, const int *g, int nrows,
                         uint32_t *out) {
  int N = c->n;
  int *e = malloc(sizeof(int) * N);
  const double sd = 3.2, mx = 6 * 3.2;
  for (int j = 0; j < N; j += 2) {
    double u1 = rng_unit(r), u2 = rng_unit(r);
    if (u1 < 1e-300) u1 = 1e-300;
    double rad = sqrt(-2.0 * log(u1));
    double v[2] = {rad * cos(2 * M_PI * u2) * sd, rad * sin(2 * M_PI * u2) * sd};
    for (int k = 0; k < 2 && j + k < N; k++) {
      double x = v[k];
      if (x > mx) x = mx;
      if (x < -mx) x = -mx;
      e[j + k] = (int)llround(x);
    }
  }
  for (int i = 0; i < nrows; i++) {
    uint32_t p = c->primes[g[i]];
    for (int j = 0; j < N; j++)
      out[(size_t)i * N + j] = e[j] < 0 ? p - (uint32_t)(-e[j]) : (uint32_t)e[j];
    orc_ntt_limb(c, g[i], out + (size_t)i * N, 1);
  }
  free(e);
}

int orc_gen_evk(const orc_ctx *c, uint64_t seed, const uint32_t *enc_s,
                const uint32_t *target_s, uint32_t *key_bx, uint32_t *key_ax) {
  /* UserInterface.cu:366-458 (PrepareEvk) over the max-level key basis */
  int N = c->n, tot = c->nprimes, L = c->L, na = c->alpha;
  int beta = (L + na - 1) / na;
  rng_t r;
  rng_seed(&r, seed);
  int g[256];
  for (int i = 0; i < tot; i++) g[i] = i;
  size_t ksz = (size_t)tot * N;
  uint32_t *e = malloc(ksz * sizeof(uint32_t));
  for (int i = 0; i < beta; i++) {
    uint32_t *kb = key_bx + i * ksz, *ka = key_ax + i * ksz;
    for (int gi = 0; gi < tot; gi++)
      for (int j = 0; j < N; j++) ka[(size_t)gi * N + j] = (uint32_t)rng_below(&r, c->primes[gi]);
    sample_error(c, &r, g, tot, e);
    for (int gi = 0; gi < tot; gi++) {
      uint32_t q = c->primes[gi];
      int32_t qi = c->qinv[gi];
      for (int j = 0; j < N; j++) {
        size_t k = (size_t)gi * N + j;
        uint32_t as = orc_mont_mult(ka[k], enc_s[k], q, qi);
        kb[k] = sub_mod(e[k], as, q);
      }
    }
    int s0 = i * na, s1 = (i + 1) * na;
    if (s1 > L) s1 = L;
    for (int gi = s0; gi < s1; gi++) {
      uint32_t q = c->primes[gi];
      int32_t qi = c->qinv[gi];
      for (int j = 0; j < N; j++) {
        size_t k = (size_t)gi * N + j;
        kb[k] = add_mod(kb[k], orc_mont_mult(target_s[k], c->p_prod[gi], q, qi), q);
      }
    }
  }
  free(e);
  return 0;
}
int orc_gen_mult_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                     uint32_t *key_bx, uint32_t *key_ax) {
  /* UserInterface.cu:329-341: target s^2 */
  size_t tot = (size_t)c->nprimes * c->n;
  uint32_t *s2 = malloc(tot * sizeof(uint32_t));
  for (int g = 0; g < c->nprimes; g++)
    for (int j = 0; j < c->n; j++) {
      size_t k = (size_t)g * c->n + j;
      s2[k] = orc_mont_mult(s[k], s[k], c->primes[g], c->qinv[g]);
    }
  int rc = orc_gen_evk(c, seed, s, s2, key_bx, key_ax);
  free(s2);
  return rc;
}
int orc_gen_rot_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                    int amount, uint32_t *key_bx, uint32_t *key_ax) {
  /* UserInterface.cu:278-316: encryption secret = s permuted by N/2 - r */
  if (amount <= 0 || amount >= c->n / 2) return -1;
  size_t tot = (size_t)c->nprimes * c->n;
  uint32_t *sr = malloc(tot * sizeof(uint32_t));
  permute_rows(c, c->nprimes, galois_of(c, c->n / 2 - amount), s, sr);
  int rc = orc_gen_evk(c, seed, sr, s, key_bx, key_ax);
  free(sr);
  return rc;
}
int orc_gen_conj_key(const orc_ctx *c, uint64_t seed, const uint32_t *s,
                     uint32_t *key_bx, uint32_t *key_ax) {
  size_t tot = (size_t)c->nprimes * c->n;
  uint32_t *sc = malloc(tot * sizeof(uint32_t));
  permute_rows(c, c->nprimes, galois_of(c, -1), s, sc);
  int rc = orc_gen_evk(c, seed, sc, s, key_bx, key_ax);
  free(sc);
  return rc;
}

int orc_encrypt(const orc_ctx *c, uint64_t seed, const uint32_t *s, int level,
                const uint32_t *pt, uint32_t *bx, uint32_t *ax) {
  /* UserInterface.cu:146-183: bx = -ax*s + m + e */
  np_t n = level_np(c, level, 0);
  int N = c->n, nq = np_q(n);
  int g[256];
  np_gidx(c, n, g);
  rng_t r;
  rng_seed(&r, seed);
  for (int i = 0; i < nq; i++)
    for (int j = 0; j < N; j++) ax[(size_t)i * N + j] = (uint32_t)rng_below(&r, c->primes[g[i]]);
  uint32_t *e = malloc((size_t)nq * N * sizeof(uint32_t));
  sample_error(c, &r, g, nq, e);
  for (int i = 0; i < nq; i++) {
    uint32_t q = c->primes[g[i]];
    int32_t qi = c->qinv[g[i]];
    const uint32_t *si = s + (size_t)g[i] * N;
    for (int j = 0; j < N; j++) {
      size_t k = (size_t)i * N + j;
      uint32_t v = orc_mont_mult(ax[k], si[j], q, qi);
      v = sub_mod(pt[k], v, q);
      bx[k] = add_mod(v, e[k], q);
    }
  }
  free(e);
  return 0;
}
int orc_decrypt(const orc_ctx *c, const uint32_t *s, int level,
                const uint32_t *bx, const uint32_t *ax, uint32_t *pt) {
  /* UserInterface.cu:185-206: pt = bx + ax*s */
  np_t n = level_np(c, level, 0);
  int N = c->n;
  int g[256];
  np_gidx(c, n, g);
  for (int i = 0; i < np_q(n); i++) {
    uint32_t q = c->primes[g[i]];
    int32_t qi = c->qinv[g[i]];
    const uint32_t *si = s + (size_t)g[i] * N;
    for (int j = 0; j < N; j++) {
      size_t k = (size_t)i * N + j;
      pt[k] = add_mod(bx[k], orc_mont_mult(si[j], ax[k], q, qi), q);
    }
  }
  return 0;
}


/* ========================================================================
 * ModUpToMax without sparse-secret encapsulation — BootContext.cpp:186-270
 * (INTTAndMultConst with mod_max_intt_const_, BootContext.cpp:93-107;
 * ModUpToMax1/2, ElementWise.cu:575-623; NTT(..., true) at the top level)
 * ====================================================================== */
int orc_modup_to_max(const orc_ctx *c, const uint32_t *bx, const uint32_t *ax,
                     uint32_t *res_bx, uint32_t *res_ax) {
  np_t b = level_np(c, -1, 0), mx = level_np(c, c->max_level, 0);
  int nb = np_q(b), N = c->n, tot = np_total(mx);
  if (nb < 1 || nb > 2) return -1;
  int gb[2], gm[256];
  np_gidx(c, b, gb);
  np_gidx(c, mx, gm);
  const uint32_t *src[2] = {bx, ax};
  uint32_t *dst[2] = {res_bx, res_ax};
  int32_t *t = malloc(sizeof(int32_t) * (size_t)nb * N);
  for (int part = 0; part < 2; part++) {
    for (int i = 0; i < nb; i++) {
      uint32_t q = c->primes[gb[i]];
      uint32_t k = (uint32_t)(N % q);
      for (int j = 0; j < nb; j++)
        if (j != i) k = mul_mod(k, c->primes[gb[j]], q);
      k = orc_inv_mod(k, q);
      int32_t *a = t + (size_t)i * N;
      memcpy(a, src[part] + (size_t)i * N, sizeof(int32_t) * N);
      intt_core(c, gb[i], a);
      for (int j = 0; j < N; j++) a[j] = ep_mult(a[j], k, q, c->qinv[gb[i]]);
    }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < tot; r++) {
      int64_t p = c->primes[gm[r]];
      uint32_t *o = dst[part] + (size_t)r * N;
      for (int j = 0; j < N; j++) {
        if (nb == 1) {
          o[j] = (uint32_t)((uint32_t)t[j] % (uint32_t)p);
        } else {
          int64_t q0 = c->primes[gb[0]], q1 = c->primes[gb[1]], qp = q0 * q1;
          int64_t v = (int64_t)(uint32_t)t[j] * q1 + (int64_t)(uint32_t)t[N + j] * q0;
          if (v >= qp) v -= qp;
          if (v > (qp >> 1)) v -= qp;
          int64_t m = v % p;
          if (m < 0) m += p;
          o[j] = (uint32_t)m;
        }
      }
      orc_ntt_limb(c, gm[r], o, 1);
    }
  }
  free(t);
  return 0;
}

/* ModUpToMax with sparse-secret encapsulation — BootContext.cpp:186-270:
 * dense-to-sparse MultKey at level -1 (Context.cpp:584-607, DtS mod switcher,
 * p_prod_dts of Context.cpp:108-123), exact lift of bx to the top-level q
 * primes and of ax to the top-level q and alpha aux primes, PMult with the
 * digit-0 sparse-to-dense key plus P * bx on the q primes (PseudoModUp,
 * CAccum), ModDown with the top level's mod switcher.  Key layouts: dts
 * [num_q(-1) + sse aux][N] (one digit), std [L + alpha][N] (digit 0). */
int orc_modup_to_max_sse(const orc_ctx *c, const uint32_t *bx, const uint32_t *ax,
                         const uint32_t *dts_bx, const uint32_t *dts_ax,
                         const uint32_t *std_bx, const uint32_t *std_ax,
                         uint32_t *res_bx, uint32_t *res_ax) {
  const msw_t *m = &c->msw[0];
  np_t b = level_np(c, -1, 0), db = level_np(c, -1, m->num_aux);
  int nb = np_q(b), dt = np_total(db), N = c->n;
  if (nb < 1 || nb > 2 || m->beta != 1) return -1;
  int gd[256];
  np_gidx(c, db, gd);
  /* 1. DtS key switch */
  uint32_t *mu = malloc(sizeof(uint32_t) * (size_t)dt * N);
  uint32_t *acc = malloc(sizeof(uint32_t) * 2 * (size_t)dt * N);
  uint32_t *sw = malloc(sizeof(uint32_t) * 2 * (size_t)nb * N);
  modup_impl(c, m, b, ax, mu);
  for (int r = 0; r < dt; r++) {
    uint32_t q = c->primes[gd[r]];
    int32_t qi = c->qinv[gd[r]];
    uint32_t pp = 1;
    for (int j = 0; j < m->num_aux; j++) pp = mul_mod(pp, c->primes[gd[nb + j]], q);
    pp = orc_to_mont(pp, q);
    for (int j = 0; j < N; j++) {
      size_t k = (size_t)r * N + j;
      uint32_t vb = orc_mont_mult(mu[k], dts_bx[k], q, qi);
      uint32_t va = orc_mont_mult(mu[k], dts_ax[k], q, qi);
      if (r < nb) vb = add_mod(vb, orc_mont_mult(bx[k], pp, q, qi), q);
      acc[k] = vb;
      acc[(size_t)dt * N + k] = va;
    }
  }
  moddown_worker(c, -1, MD_MODDOWN, acc, sw);
  moddown_worker(c, -1, MD_MODDOWN, acc + (size_t)dt * N, sw + (size_t)nb * N);
  /* 2. lift */
  np_t top = level_np(c, c->max_level, 0), tqp = level_np(c, c->max_level, c->alpha);
  int nq = np_q(top), qt = np_total(tqp);
  int gb[2], gm[256];
  np_gidx(c, b, gb);
  np_gidx(c, tqp, gm);
  int32_t *t = malloc(sizeof(int32_t) * 2 * (size_t)nb * N);
  for (int part = 0; part < 2; part++)
    for (int i = 0; i < nb; i++) {
      uint32_t q = c->primes[gb[i]];
      uint32_t k = (uint32_t)(N % q);
      for (int j = 0; j < nb; j++)
        if (j != i) k = mul_mod(k, c->primes[gb[j]], q);
      k = orc_inv_mod(k, q);
      int32_t *a = t + ((size_t)part * nb + i) * N;
      memcpy(a, sw + ((size_t)part * nb + i) * N, sizeof(int32_t) * N);
      intt_core(c, gb[i], a);
      for (int j = 0; j < N; j++) a[j] = ep_mult(a[j], k, q, c->qinv[gb[i]]);
    }
  uint32_t *lb = malloc(sizeof(uint32_t) * (size_t)nq * N);
  uint32_t *la = malloc(sizeof(uint32_t) * (size_t)qt * N);
  for (int part = 0; part < 2; part++) {
    int rows = part == 0 ? nq : qt;
    uint32_t *o = part == 0 ? lb : la;
    const int32_t *src = t + (size_t)part * nb * N;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; r++) {
      int64_t p = c->primes[gm[r]];
      uint32_t *row = o + (size_t)r * N;
      for (int j = 0; j < N; j++) {
        if (nb == 1) {
          row[j] = (uint32_t)((uint32_t)src[j] % (uint32_t)p);
        } else {
          int64_t q0 = c->primes[gb[0]], q1 = c->primes[gb[1]], qp = q0 * q1;
          int64_t v = (int64_t)(uint32_t)src[j] * q1 + (int64_t)(uint32_t)src[N + j] * q0;
          if (v >= qp) v -= qp;
          if (v > (qp >> 1)) v -= qp;
          int64_t mm = v % p;
          if (mm < 0) mm += p;
          row[j] = (uint32_t)mm;
        }
      }
      orc_ntt_limb(c, gm[r], row, 1);
    }
  }
  /* 3. StD: key digit 0 (.) a_lift + P * b_lift on q primes; ModDown */
  int po = c->max_ter - top.num_ter;
  uint32_t *acc2 = malloc(sizeof(uint32_t) * 2 * (size_t)qt * N);
  for (int r = 0; r < qt; r++) {
    uint32_t q = c->primes[gm[r]];
    int32_t qi = c->qinv[gm[r]];
    int kr = r < nq ? po + r : c->L + (r - nq);
    for (int j = 0; j < N; j++) {
      size_t k = (size_t)r * N + j, kk = (size_t)kr * N + j;
      uint32_t vb = orc_mont_mult(la[k], std_bx[kk], q, qi);
      uint32_t va = orc_mont_mult(la[k], std_ax[kk], q, qi);
      if (r < nq) vb = add_mod(vb, orc_mont_mult(lb[k], c->p_prod[po + r], q, qi), q);
      acc2[k] = vb;
      acc2[(size_t)qt * N + k] = va;
    }
  }
  moddown_worker(c, c->max_level, MD_MODDOWN, acc2, res_bx);
  moddown_worker(c, c->max_level, MD_MODDOWN, acc2 + (size_t)qt * N, res_ax);
  free(mu);
  free(acc);
  free(sw);
  free(t);
  free(lb);
  free(la);
  free(acc2);
  return 0;
}

/* ---- encoding — Encode.cpp:10-21, 84-133, 135-190, 250-275 ---- */
typedef struct {
  double re, im;
} cplx;
static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static void bitrev_cplx(cplx *d, int n) {
  int lb = 0;
  while ((1 << lb) < n) lb++;
  for (int i = 0; i < n; i++) {
    int j = (int)brev((unsigned)i, lb);
    if (i < j) {
      cplx t = d[i];
      d[i] = d[j];
      d[j] = t;
    }
  }
}
static void special_ifft(const orc_ctx *c, cplx *d, int ns) {
  int M = 2 * c->n;
  for (int stride = ns / 2; stride >= 1; stride /= 2) {
    int sg = stride * 2, st8 = stride << 3, gap = M / st8;
    for (int i = 0; i < ns; i += sg)
      for (int j = 0; j < stride; j++) {
        int ti = (st8 - (c->galois[j] % st8)) * gap;
        cplx w = {cos(2.0 * M_PI * ti / M), sin(2.0 * M_PI * ti / M)};
        cplx x = {d[i + j].re + d[i + j + stride].re, d[i + j].im + d[i + j + stride].im};
        cplx y = {d[i + j].re - d[i + j + stride].re, d[i + j].im - d[i + j + stride].im};
        y = cmul(y, w);
        d[i + j] = x;
        d[i + j + stride] = y;
      }
  }
  bitrev_cplx(d, ns);
  for (int i = 0; i < ns; i++) {
    d[i].re /= ns;
    d[i].im /= ns;
  }
}
static void special_fft(const orc_ctx *c, cplx *d, int ns) {
  int M = 2 * c->n;
  bitrev_cplx(d, ns);
  for (int stride = 1; stride < ns; stride *= 2) {
    int sg = stride * 2, st8 = stride << 3, gap = M / st8;
    for (int i = 0; i < ns; i += sg)
      for (int j = 0; j < stride; j++) {
        int ti = (c->galois[j] % st8) * gap;
        cplx w = {cos(2.0 * M_PI * ti / M), sin(2.0 * M_PI * ti / M)};
        cplx x = d[i + j], y = cmul(d[i + j + stride], w);
        d[i + j].re = x.re + y.re;
        d[i + j].im = x.im + y.im;
        d[i + j + stride].re = x.re - y.re;
        d[i + j + stride].im = x.im - y.im;
      }
  }
}
/* BigInt(double) truncates toward zero; result mod p in [0, p). */
static uint32_t double_mod(double v, uint32_t p) {
  if (v == 0.0) return 0;
  int neg = v < 0;
  double a = fabs(v);
  uint64_t r;
  if (a < 18446744073709551616.0) {
    uint64_t t = (uint64_t)a;
    r = t % p;
  } else {
    int e;
    double m = frexp(a, &e); /* a = m * 2^e, m in [0.5, 1) */
    uint64_t mi = (uint64_t)ldexp(m, 53);
    int sh = e - 53;
    uint64_t pw = 1 % p, b = 2;
    while (sh) {
      if (sh & 1) pw = (pw * b) % p;
      b = (b * b) % p;
      sh >>= 1;
    }
    r = ((mi % p) * pw) % p;
  }
  if (neg && r) r = p - r;
  return (uint32_t)r;
}
int orc_encode(const orc_ctx *c, int level, double scale, const double *re,
               const double *im, int num_slots, int num_aux, uint32_t *pt) {
  int N = c->n, half = N / 2;
  if (num_slots < 1 || num_slots > half || (num_slots & (num_slots - 1))) return -1;
  np_t n = level_np(c, level, num_aux);
  int g[256];
  np_gidx(c, n, g);
  cplx *d = malloc(sizeof(cplx) * num_slots);
  for (int i = 0; i < num_slots; i++) {
    d[i].re = re[i];
    d[i].im = im[i];
  }
  special_ifft(c, d, num_slots);
  int gap = half / num_slots, tot = np_total(n);
  memset(pt, 0, sizeof(uint32_t) * (size_t)tot * N);
  for (int i = 0; i < num_slots; i++) {
    double vr = d[i].re * scale, vi = d[i].im * scale;
    for (int k = 0; k < tot; k++) {
      uint32_t p = c->primes[g[k]];
      pt[(size_t)k * N + i * gap] = double_mod(vr, p);
      pt[(size_t)k * N + i * gap + half] = double_mod(vi, p);
    }
  }
  free(d);
  for (int k = 0; k < tot; k++) orc_ntt_limb(c, g[k], pt + (size_t)k * N, 1);
  return 0;
}
int orc_encode_const(const orc_ctx *c, int level, double scale, double value,
                     int num_aux, uint32_t *cx) {
  np_t n = level_np(c, level, num_aux);
  int g[256];
  np_gidx(c, n, g);
  double v = value * scale;
  for (int k = 0; k < np_total(n); k++) {
    uint32_t p = c->primes[g[k]];
    cx[k] = orc_to_mont(double_mod(v, p), p);
  }
  return 0;
}
int orc_decode(const orc_ctx *c, int level, double scale, const uint32_t *pt,
               int num_slots, double *re, double *im) {
  /* Encode.cpp:45-82 + 192-248.  The coefficient is recovered by CRT over the
   * first primes whose product exceeds 2^100 (exact for any coefficient of
   * magnitude below that), which equals the full-basis centred CRT for every
   * decryptable plaintext. */
  int N = c->n, half = N / 2;
  np_t n = level_np(c, level, 0);
  int g[256];
  np_gidx(c, n, g);
  int nq = np_q(n);
  int K = 0;
  double lg = 0;
  while (K < nq && lg < 100.0) {
    lg += log2((double)c->primes[g[K]]);
    K++;
  }
  if (lg > 124.0) { /* keep the CRT product below 2^126 */
    K--;
  }
  uint32_t *co = malloc(sizeof(uint32_t) * (size_t)K * N);
  for (int k = 0; k < K; k++) {
    memcpy(co + (size_t)k * N, pt + (size_t)k * N, sizeof(uint32_t) * N);
    orc_intt_limb(c, g[k], co + (size_t)k * N, 1);
  }
  /* Garner with __int128 */
  unsigned __int128 Q = 1;
  for (int k = 0; k < K; k++) Q *= c->primes[g[k]];
  unsigned __int128 hQ = Q / 2;
  cplx *d = malloc(sizeof(cplx) * num_slots);
  int gap = half / num_slots;
  for (int i = 0; i < num_slots; i++) {
    for (int part = 0; part < 2; part++) {
      int idx = i * gap + part * half;
      unsigned __int128 x = co[idx] % c->primes[g[0]], prod = c->primes[g[0]];
      for (int k = 1; k < K; k++) {
        uint32_t p = c->primes[g[k]];
        uint64_t xm = (uint64_t)(x % p);
        uint64_t pm = (uint64_t)(prod % p);
        uint64_t diff = (co[(size_t)k * N + idx] + p - xm) % p;
        uint64_t t = (diff * orc_inv_mod((uint32_t)pm, p)) % p;
        x += prod * t;
        prod *= p;
      }
      double v = x > hQ ? -(double)(Q - x) : (double)x;
      v /= scale;
      if (part == 0)
        d[i].re = v;
      else
        d[i].im = v;
    }
  }
  free(co);
  special_fft(c, d, num_slots);
  for (int i = 0; i < num_slots; i++) {
    re[i] = d[i].re;
    im[i] = d[i].im;
  }
  free(d);
  return 0;
}

/* Per-level ModSwitch constants (for comparison with the CUDA library's host
 * code): kind 0 = ModUp digit, 1 = ModDown, 2 = Rescale, 3 = ModDown+Rescale;
 * dims = {K, M, pad_len, restore_start, restore_end, beta}. */
int orc_level_consts(const orc_ctx *c, int level, int kind, int digit,
                     uint32_t *c1, int32_t *table, uint32_t *inv,
                     uint32_t *pad, int *dims) {
  if (level < -1 || level > c->max_level) return -1;
  const msw_t *m = &c->msw[level + 1];
  int K = 0, M = 0, pl = 0;
  dims[3] = m->restore_start;
  dims[4] = m->restore_end;
  dims[5] = m->beta;
  const uint32_t *v1 = NULL, *vi = NULL, *vp = NULL;
  const int32_t *vt = NULL;
  if (kind == 0) {
    if (digit < 0 || digit >= m->beta) return -1;
    K = m->dig_e[digit] - m->dig_s[digit];
    if (m->dig_e[digit] <= 0) K = 0;
    if (K <= 0) {
      dims[0] = dims[1] = dims[2] = 0;
      return 0;
    }
    M = m->num_q + m->num_aux - K;
    v1 = m->mod_up1 + m->dig_s[digit];
    vt = m->mod_up2[digit];
  } else if (kind == 1) {
    K = m->num_aux;
    M = m->num_q;
    v1 = m->mod_down1;
    vt = m->mod_down2;
    vi = m->inv_p_prod;
  } else if (kind == 2 || kind == 3) {
    if (!m->has_rescale) return -1;
    K = kind == 2 ? m->rs_src_len : m->mdr_src_len;
    M = m->rs_dst_len;
    pl = M - (m->restore_end - m->restore_start);
    v1 = kind == 2 ? m->rs1 : m->mdr1;
    vt = kind == 2 ? m->rs2 : m->mdr2;
    vi = kind == 2 ? m->rs_inv : m->mdr_inv;
    vp = kind == 2 ? m->rs_pad : m->mdr_pad;
  } else {
    return -1;
  }
  dims[0] = K;
  dims[1] = M;
  dims[2] = pl;
  if (v1 && c1) memcpy(c1, v1, sizeof(uint32_t) * K);
  if (vt && table) memcpy(table, vt, sizeof(int32_t) * (size_t)K * M);
  if (vi && inv) memcpy(inv, vi, sizeof(uint32_t) * M);
  if (vp && pad) memcpy(pad, vp, sizeof(uint32_t) * pl);
  return 0;
}
