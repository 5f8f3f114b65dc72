// Host side of the bootstrapping path: constants for the linear transforms
// and EvalMod (Encoder::EncodeConstant: value * scale truncated toward zero
// to an integer, BigInt(double) of include/core/BigInt.h:24, then residues),
// the encoder's twiddle table, and ModUpToMax.  The plaintext encoder and
// the decoder run on the device (codec.cu).
#include <cmath>
#include <complex>

#include "host.h"
#include "kernels.h"

namespace chd {
namespace {

using cd = std::complex<double>;

// round-toward-zero integer of v, reduced to [0, p): exact for every finite
// double (|v| >= 2^53 is already an integer m * 2^e)
uint32_t trunc_mod(double v, uint32_t p) {
  if (v == 0.0) return 0;
  const bool neg = v < 0;
  const double a = std::fabs(v);
  uint64_t r;
  if (a < 18446744073709551616.0) {
    r = static_cast<uint64_t>(a) % p;
  } else {
    int e;
    const double m = std::frexp(a, &e);  // a = m 2^e, m in [0.5, 1)
    const uint64_t mi = static_cast<uint64_t>(std::ldexp(m, 53));
    uint64_t pw = 1 % p, b = 2;
    for (int sh = e - 53; sh; sh >>= 1) {
      if (sh & 1) pw = pw * b % p;
      b = b * b % p;
    }
    r = (mi % p) * pw % p;
  }
  if (neg && r) r = p - r;
  return static_cast<uint32_t>(r);
}

}  // namespace

// BootParameter's EvalMod polynomial (src/extension/BootParameter.cpp:13-23):
// Chebyshev coefficients of the cosine approximation, to be used with
// initial K = 2 and three double-angle steps.  The values are the
// reference's, digit for digit, because the encoded constants (and hence
// every residue of a bootstrap) depend on them.
const std::vector<double> &boot_mod_coefficients() {
  static const std::vector<double> c{
      0.12517186708929745802,    0.0, 0.2894364973331168731,      0.0,
      0.36272381596524499154,    0.0, 0.3011054704600794278,      0.0,
      -0.10550875667295944105,   0.0, -0.43588877795190139706,    0.0,
      0.37482647434055190702,    0.0, -0.14821069913569220404,    0.0,
      0.03665437786710548091,    0.0, -0.0063882548960017121343,  0.0,
      0.00083684232451067872756, 0.0, -8.6443599931576702305e-05, 0.0,
      7.0966437900548814324e-06, 0.0, -5.228015817181348194e-07,  0.0,
      2.2714690137973883081e-08, 0.0, -2.3761936068138980797e-09};
  return c;
}

const std::vector<std::complex<double>> &Context::enc_twiddles() {
  if (enc_tw.empty()) {
    const int M = 2 * P->n;
    enc_tw.resize(M);
    for (int i = 0; i < M; i++) enc_tw[i] = std::polar(1.0, 2.0 * M_PI * i / M);
  }
  return enc_tw;
}

void Context::encode_const(int level, double scale, double value, int num_aux, std::vector<uint32_t> *cx) const {
  // Encoder::EncodeConstant, Encode.cpp:250-275
  const NP np = P->level_np(level, num_aux);
  const int tot = np.total();
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  cx->resize(tot);
  const double v = value * scale;
  for (int k = 0; k < tot; k++) {
    const uint32_t p = P->primes[g[k]];
    (*cx)[k] = prime::to_mont(trunc_mod(v, p), p);
  }
}

Status Context::modup_to_max(DeviceCt &res, const DeviceCt &a) {
  // BootContext::ModUpToMax without sparse-secret encapsulation
  // (BootContext.cpp:186-270): per part, INTTAndMultConst with
  // (prod_{j != i} q_j * N)^-1 (BootContext.cpp:93-107), the CRT lift
  // (ElementWise.cu:575-623, 1646-1670), NTT to the top level.
  const NP np = P->level_np(-1);
  CHD_CHECK(a.np == np, kErrShape, "ModUpToMax: input must be at level -1 without aux primes");
  CHD_CHECK(!a.has_rx, kErrShape, "ModUpToMax: input has Rx");
  const int nb = np.q();
  CHD_CHECK(nb == 1 || nb == 2, kErrUnsupported, "ModUpToMax: level -1 must have one or two primes");
  const int n = P->n;
  int g[2];
  P->gidx(np, g);
  ArenaScope scope(arena);
  uint32_t *t = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(2) * nb * n * 4));
  CHD_CHECK(t, kErrAlloc, "ModUpToMax: scratch allocation failed");
  RowBatch rb;
  rb.count = 0;
  for (int part = 0; part < 2; part++)
    for (int i = 0; i < nb; i++) {
      const uint32_t q = P->primes[g[i]];
      uint32_t c = static_cast<uint32_t>(n % q);
      for (int j = 0; j < nb; j++)
        if (j != i) c = prime::mul_mod(c, P->primes[g[j]], q);
      c = prime::inv_mod(c, q);  // plain, applied like a Montgomery constant
      RowDesc &d = rb.rows[rb.count++];
      d = RowDesc{};
      d.src = (part == 0 ? a.bx : a.ax) + static_cast<size_t>(i) * n;
      d.dst = t + (static_cast<size_t>(part) * nb + i) * n;
      d.tw = itw(g[i]);
      d.q = q;
      mont_as_shoup(c, g[i], &d.c0, &d.c0s);
    }
  launch_ntt_inv(rb, P->log_n, stream);
  const NP maxnp = P->level_np(P->max_level);
  const double scale = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(maxnp, false, n));
  ModUpToMaxDesc d{};
  d.src[0] = t;
  d.src[1] = t + static_cast<size_t>(nb) * n;
  d.dst[0] = res.bx;
  d.dst[1] = res.ax;
  std::vector<int> gm(maxnp.total());
  P->gidx(maxnp, gm.data());
  for (int r = 0; r < maxnp.total(); r++) d.p[r] = P->primes[gm[r]];
  d.q0 = P->primes[g[0]];
  d.q1 = nb == 2 ? P->primes[g[1]] : 0;
  d.nbase = nb;
  d.rows = maxnp.total();
  d.parts = 2;
  d.n = n;
  launch_modup_to_max(d, stream);
  CHD_TRY(ntt(maxnp, res.bx, true));
  CHD_TRY(ntt(maxnp, res.ax, true));
  res.scale = scale;
  res.num_slots = slots;
  return check_cuda("ModUpToMax");
}

Status Context::modup_to_max_sse(DeviceCt &res, const DeviceCt &a, const DeviceEvk &dts, const DeviceEvk &std_key) {
  // BootContext::ModUpToMax with sparse-secret encapsulation
  // (BootContext.cpp:186-270):
  //   1. dense-to-sparse key switch at level -1 (MultKey with the DtS mod
  //      switcher, Context.cpp:584-607 / 650-712): ModUp(a) (.) key +
  //      P_dts b, ModDown, over the level -1 primes and sse aux primes;
  //   2. both parts lifted exactly to the top level, a also to the alpha
  //      auxiliary primes (INTTAndMultConst, ModUpToMax, NTT);
  //   3. sparse-to-dense key switch with the single-digit key:
  //      (key (.) a_lift + (P b_lift, 0)), ModDown at the top level.
  const NP np = P->level_np(-1);
  CHD_CHECK(a.np == np && !a.has_rx, kErrShape, "ModUpToMax: input must be at level -1 without Rx");
  const LevelMS &m = lms(-1);
  const int nb = np.q(), na = m.num_aux, n = P->n;
  const NP dnp = P->level_np(-1, na);
  CHD_CHECK(dts.np == dnp && dts.beta >= 1, kErrKey, "ModUpToMax: dense-to-sparse key basis mismatch");
  CHD_CHECK(std_key.np.aux == P->alpha && std_key.np.q() == P->L, kErrKey,
            "ModUpToMax: sparse-to-dense key basis mismatch");
  CHD_CHECK(m.beta == 1, kErrUnsupported, "ModUpToMax: level -1 key switch must have one digit");
  ArenaScope scope(arena);
  const size_t N = static_cast<size_t>(n);
  // 1. DtS key switch
  const int dtot = dnp.total();
  std::vector<int> gd(dtot);
  P->gidx(dnp, gd.data());
  uint32_t *mu = static_cast<uint32_t *>(arena.alloc(dtot * N * 4));
  uint32_t *acc = static_cast<uint32_t *>(arena.alloc(2 * dtot * N * 4));
  uint32_t *sw = static_cast<uint32_t *>(arena.alloc(2 * nb * N * 4));
  CHD_CHECK(mu && acc && sw, kErrAlloc, "ModUpToMax: scratch allocation failed");
  uint32_t *mus[1] = {mu};
  CHD_TRY(modup(-1, a.ax, mus));
  {
    KeyMacDesc d{};
    d.kb[0] = dts.bx;
    d.ka[0] = dts.ax;
    d.beta = 1;
    d.rows = dtot;
    d.nq = nb;
    d.count = 1;
    for (int r = 0; r < dtot; r++) {
      const uint32_t q = P->primes[gd[r]];
      d.q[r] = q;
      d.qinv[r] = P->qinv[gd[r]];
      d.key_row[r] = static_cast<int16_t>(r);
      if (r < nb) {
        uint32_t v = 1;
        for (int j = 0; j < na; j++) v = prime::mul_mod(v, P->primes[gd[nb + j]], q);
        d.p_prod[r] = prime::to_mont(v, q);  // p_prod_dts, Context.cpp:108-123
      }
    }
    d.ct[0].mu[0] = mu;
    d.ct[0].d0 = a.bx;
    d.ct[0].d1 = nullptr;
    d.ct[0].acc_b = acc;
    d.ct[0].acc_a = acc + dtot * N;
    launch_key_mac(d, P->log_n, stream);
  }
  {
    const uint32_t *src[2] = {acc, acc + dtot * N};
    uint32_t *dst[2] = {sw, sw + nb * N};
    CHD_TRY(moddown(-1, MDType::kModDown, src, dst, 2));
  }
  // 2. lift: b to the top-level q primes, a to the top-level q and aux primes
  int g[2];
  P->gidx(np, g);
  uint32_t *t = static_cast<uint32_t *>(arena.alloc(2 * nb * N * 4));
  CHD_CHECK(t, kErrAlloc, "ModUpToMax: scratch allocation failed");
  RowBatch rb;
  rb.count = 0;
  for (int part = 0; part < 2; part++)
    for (int i = 0; i < nb; i++) {
      const uint32_t q = P->primes[g[i]];
      uint32_t c = static_cast<uint32_t>(n % q);
      for (int j = 0; j < nb; j++)
        if (j != i) c = prime::mul_mod(c, P->primes[g[j]], q);
      c = prime::inv_mod(c, q);
      RowDesc &d = rb.rows[rb.count++];
      d = RowDesc{};
      d.src = sw + (static_cast<size_t>(part) * nb + i) * N;
      d.dst = t + (static_cast<size_t>(part) * nb + i) * N;
      d.tw = itw(g[i]);
      d.q = q;
      mont_as_shoup(c, g[i], &d.c0, &d.c0s);
    }
  launch_ntt_inv(rb, P->log_n, stream);
  const NP top = P->level_np(P->max_level);
  const NP topqp = P->level_np(P->max_level, P->alpha);
  const int nq = top.q(), qtot = topqp.total();
  uint32_t *lb = static_cast<uint32_t *>(arena.alloc(nq * N * 4));
  uint32_t *la = static_cast<uint32_t *>(arena.alloc(qtot * N * 4));
  CHD_CHECK(lb && la, kErrAlloc, "ModUpToMax: scratch allocation failed");
  std::vector<int> gm(qtot);
  P->gidx(topqp, gm.data());
  for (int part = 0; part < 2; part++) {
    ModUpToMaxDesc d{};
    d.src[0] = t + static_cast<size_t>(part) * nb * N;
    d.dst[0] = part == 0 ? lb : la;
    d.rows = part == 0 ? nq : qtot;
    for (int r = 0; r < d.rows; r++) d.p[r] = P->primes[gm[r]];
    d.q0 = P->primes[g[0]];
    d.q1 = nb == 2 ? P->primes[g[1]] : 0;
    d.nbase = nb;
    d.parts = 1;
    d.n = n;
    launch_modup_to_max(d, stream);
  }
  CHD_TRY(ntt(top, lb, true));
  CHD_TRY(ntt(topqp, la, true));
  // 3. StD key switch with the digit-0 key, then ModDown at the top level
  uint32_t *acc2 = static_cast<uint32_t *>(arena.alloc(2 * qtot * N * 4));
  CHD_CHECK(acc2, kErrAlloc, "ModUpToMax: scratch allocation failed");
  {
    KeyMacDesc d{};
    d.kb[0] = std_key.bx;
    d.ka[0] = std_key.ax;
    d.beta = 1;
    d.rows = qtot;
    d.nq = nq;
    d.count = 1;
    const int prime_offset = P->max_ter - top.ter;
    for (int r = 0; r < qtot; r++) {
      d.q[r] = P->primes[gm[r]];
      d.qinv[r] = P->qinv[gm[r]];
      d.key_row[r] = static_cast<int16_t>(r < nq ? prime_offset + r : P->L + (r - nq));
      d.p_prod[r] = r < nq ? p_prod[prime_offset + r] : 0;
    }
    d.ct[0].mu[0] = la;
    d.ct[0].d0 = lb;
    d.ct[0].d1 = nullptr;
    d.ct[0].acc_b = acc2;
    d.ct[0].acc_a = acc2 + qtot * N;
    launch_key_mac(d, P->log_n, stream);
  }
  const double scale = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(top, false, n));
  {
    const uint32_t *src[2] = {acc2, acc2 + qtot * N};
    uint32_t *dst[2] = {res.bx, res.ax};
    CHD_TRY(moddown(P->max_level, MDType::kModDown, src, dst, 2));
  }
  res.scale = scale;
  res.num_slots = slots;
  return check_cuda("ModUpToMax (sparse-secret encapsulation)");
}

}  // namespace chd
