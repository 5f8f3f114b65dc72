// Host side of the 64-bit word path (w64.h): prime utilities, the level
// model, ModSwitch constants, the evaluation core and its C ABI (chd64_*).
// Each routine is the 32-bit path's restatement of the reference with
// word = uint64_t and R = 2^64; 128-bit host arithmetic replaces the 64-bit
// intermediates.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/cheddar_b200.h"
#include "w64.h"

namespace chd {
namespace w64 {

// ------------------------------------------------------------ primes
u64 mul_mod(u64 a, u64 b, u64 q) { return static_cast<u64>(static_cast<u128>(a) * b % q); }

u64 inv_mod(u64 a, u64 q) {
  i128 t = 0, nt = 1, r = q, nr = a % q;
  while (nr) {
    const i128 k = r / nr;
    i128 tmp = t - k * nt;
    t = nt;
    nt = tmp;
    tmp = r - k * nr;
    r = nr;
    nr = tmp;
  }
  if (t < 0) t += q;
  return static_cast<u64>(t);
}

u64 pow_mod(u64 a, int64_t e, u64 q) {
  a %= q;
  if (e < 0) {
    a = inv_mod(a, q);
    e = -e;
  }
  u64 r = 1;
  while (e) {
    if (e & 1) r = mul_mod(r, a, q);
    a = mul_mod(a, a, q);
    e >>= 1;
  }
  return r;
}

namespace {
// deterministic Miller-Rabin for 64-bit integers
bool is_prime64(u64 n) {
  if (n < 2) return false;
  for (u64 p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    if (n % p == 0) return n == p;
  }
  u64 d = n - 1;
  int s = 0;
  while (!(d & 1)) {
    d >>= 1;
    s++;
  }
  for (u64 a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    u64 x = pow_mod(a, static_cast<int64_t>(d), n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s && comp; r++) {
      x = mul_mod(x, x, n);
      if (x == n - 1) comp = false;
    }
    if (comp) return false;
  }
  return true;
}
u64 gcd64(u64 a, u64 b) {
  while (b) {
    const u64 t = a % b;
    a = b;
    b = t;
  }
  return a;
}
// Pollard's rho (Brent's cycle detection) for a composite n
u64 rho(u64 n) {
  if (n % 2 == 0) return 2;
  for (u64 c = 1;; c++) {
    u64 x = 2, y = 2, d = 1;
    auto f = [&](u64 v) { return static_cast<u64>((static_cast<u128>(v) * v + c) % n); };
    while (d == 1) {
      x = f(x);
      y = f(f(y));
      d = gcd64(x > y ? x - y : y - x, n);
    }
    if (d != n) return d;
  }
}
void factor(u64 n, std::vector<u64> *out) {
  if (n == 1) return;
  if (is_prime64(n)) {
    out->push_back(n);
    return;
  }
  for (u64 p = 2; p < 1000; p++)
    if (n % p == 0) {
      out->push_back(p);
      while (n % p == 0) n /= p;
      factor(n, out);
      return;
    }
  const u64 d = rho(n);
  factor(d, out);
  factor(n / d, out);
}
}  // namespace

u64 smallest_generator(u64 q) {
  // the smallest r >= 2 of order q - 1 (PrimeUtils.h:135-181): the prime
  // factors of q - 1 come from Pollard's rho instead of trial division, the
  // same set, hence the same generator
  const u64 phi = q - 1;
  std::vector<u64> f;
  factor(phi, &f);
  std::sort(f.begin(), f.end());
  f.erase(std::unique(f.begin(), f.end()), f.end());
  for (u64 r = 2; r < q; r++) {
    bool ok = true;
    for (u64 x : f)
      if (pow_mod(r, static_cast<int64_t>(phi / x), q) == 1) {
        ok = false;
        break;
      }
    if (ok) return r;
  }
  return 0;
}

u64 primitive_root(u64 m, u64 q) { return pow_mod(smallest_generator(q), static_cast<int64_t>((q - 1) / m), q); }

i64 inv_mod_word(u64 q) {
  u64 x = q;
  for (int i = 0; i < 6; i++) x *= 2u - q * x;
  return static_cast<i64>(x);
}

u64 to_mont(u64 a, u64 q) { return static_cast<u64>((static_cast<u128>(a) << 64) % q); }

i64 centre(u64 a, u64 q) { return a > (q >> 1) ? static_cast<i64>(a) - static_cast<i64>(q) : static_cast<i64>(a); }

// ------------------------------------------------------------ params
namespace {
bool np_less(std::pair<int, int> a, std::pair<int, int> b) {
  const int at = a.first + a.second, bt = b.first + b.second;
  return at < bt || (at == bt && a.first < b.first);
}
unsigned brev(unsigned x, int bits) {
  unsigned r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}
}  // namespace

std::unique_ptr<Params64> Params64::create(const ParamSpec64 &spec, std::string *err) {
  // Parameter.cu:36-84 with word = uint64_t (primes below 2^62)
  if (spec.log_degree != 16) {
    *err = "the 64-bit word path supports log_degree 16";
    return nullptr;
  }
  if (spec.main_primes.empty() || spec.aux_primes.empty() || spec.level_config.empty()) {
    *err = "main_primes, auxiliary_primes and level_config must be non-empty";
    return nullptr;
  }
  const u64 two_n = 2ull << spec.log_degree;
  for (auto *lst : {&spec.main_primes, &spec.aux_primes, &spec.ter_primes})
    for (u64 p : *lst) {
      if (p >= (1ull << 62)) {
        *err = "Max prime is too large for the word size";
        return nullptr;
      }
      if (p % two_n != 1) {
        *err = "Prime is not NTT-friendly";
        return nullptr;
      }
    }
  const int nm = static_cast<int>(spec.main_primes.size()), nt = static_cast<int>(spec.ter_primes.size());
  const int na = static_cast<int>(spec.aux_primes.size());
  if (nm + nt + na > 64) {
    *err = "too many primes: at most 64 (main + terminal + auxiliary) are supported";
    return nullptr;
  }
  std::pair<int, int> prev{0, 0};
  for (size_t i = 0; i + 1 < spec.level_config.size(); i++) {
    auto c = spec.level_config[i];
    if (c.first < 0 || c.first > nm || c.second < 0 || c.second > nt || !np_less(prev, c)) {
      *err = "Invalid level configuration at level " + std::to_string(i);
      return nullptr;
    }
    prev = c;
  }
  if (spec.level_config.back() != std::make_pair(nm, nt)) {
    *err = "Invalid number of primes at the last level";
    return nullptr;
  }
  auto P = std::make_unique<Params64>();
  P->spec = spec;
  P->log_n = spec.log_degree;
  P->n = 1 << spec.log_degree;
  P->max_ter = nt;
  P->max_main = nm;
  P->L = nm + nt;
  P->alpha = na;
  P->max_level = static_cast<int>(spec.level_config.size()) - 1;
  P->short_np.main = spec.level_config[0].first - spec.additional_base.first;
  P->short_np.ter = spec.level_config[0].second - spec.additional_base.second;
  for (int i = nt - 1; i >= 0; i--) P->primes.push_back(spec.ter_primes[i]);
  for (u64 p : spec.main_primes) P->primes.push_back(p);
  for (u64 p : spec.aux_primes) P->primes.push_back(p);
  for (u64 p : P->primes) P->qinv.push_back(inv_mod_word(p));
  P->rescale_prod.assign(P->max_level + 1, 0.0);
  for (int i = 1; i <= P->max_level; i++) {
    NP up = P->level_np(i), lo = P->level_np(i - 1);
    const int td = up.ter - lo.ter, md = up.main - lo.main;
    double num = 1.0, den = 1.0;
    if (td >= 0)
      for (int j = 0; j < td; j++) num *= static_cast<double>(spec.ter_primes[lo.ter + j]);
    else
      for (int j = 0; j < -td; j++) den *= static_cast<double>(spec.ter_primes[up.ter + j]);
    if (md >= 0)
      for (int j = 0; j < md; j++) num *= static_cast<double>(spec.main_primes[lo.main + j]);
    else
      for (int j = 0; j < -md; j++) den *= static_cast<double>(spec.main_primes[up.main + j]);
    P->rescale_prod[i] = num / den;
  }
  // scales, Parameter.cu:145-190: the geometric mean of the level below's
  // scale and the rescale prime product, up to the default encryption level
  P->scale.assign(spec.default_encryption_level + 1, 0.0);
  if (!P->scale.empty()) P->scale[0] = spec.base_scale;
  for (int i = 1; i <= spec.default_encryption_level && i <= P->max_level; i++)
    P->scale[i] = std::sqrt(P->scale[i - 1] * P->rescale_prod[i]);
  return P;
}

NP Params64::level_np(int level, int num_aux) const {
  if (level == -1) return NP{short_np.main, short_np.ter, num_aux};
  auto c = spec.level_config.at(level);
  return NP{c.first, c.second, num_aux};
}

int Params64::np_to_level(const NP &np) const {
  for (int l = 0; l <= max_level; l++)
    if (spec.level_config[l].first == np.main && spec.level_config[l].second == np.ter) return l;
  return -2;
}

void Params64::gidx(const NP &np, int *out) const {
  int k = 0;
  for (int i = 0; i < np.q(); i++) out[k++] = max_ter - np.ter + i;
  for (int a = 0; a < np.aux; a++) out[k++] = L + a;
}

u64 Params64::galois_of(int amount) const {
  if (amount == -1) return 2ull * n - 1;
  u64 g = 1;
  for (int i = 0; i < amount; i++) g = g * 5 % (2ull * n);
  return g;
}

// ------------------------------------------------------------ constants
namespace {
// ModSwitch.cu:320-370 (word = uint64_t)
void ms_consts(u64 n, const std::vector<u64> &src, const std::vector<u64> &dst, int rs, int re, std::vector<u64> *c1,
               std::vector<i64> *c2) {
  const size_t sl = src.size(), dl = dst.size();
  c1->assign(sl, 1);
  c2->assign(sl * dl, 0);
  for (size_t i = 0; i < sl; i++) {
    const u64 m = src[i];
    u64 v = 1;
    for (size_t j = 0; j < sl; j++)
      if (j != i) v = mul_mod(v, src[j], m);
    v = inv_mod(mul_mod(v, n, m), m);
    for (int j = rs; j < re; j++) v = mul_mod(v, dst[j], m);
    (*c1)[i] = v;
  }
  for (size_t mi = 0; mi < dl; mi++) {
    const u64 p = dst[mi];
    for (size_t i = 0; i < sl; i++) {
      u64 acc = 1;
      for (size_t j = 0; j < sl; j++)
        if (j != i) acc = mul_mod(acc, src[j], p);
      acc = to_mont(to_mont(acc, p), p);
      (*c2)[mi * sl + i] = centre(acc, p);
    }
  }
}
// ModSwitch.cu:372-411
void epi_consts(const std::vector<u64> &src, const std::vector<u64> &dst, int rs, int re, std::vector<u64> *inv,
                std::vector<u64> *pad) {
  const size_t dl = dst.size();
  inv->assign(dl, 0);
  for (size_t i = 0; i < dl; i++) {
    const u64 p = dst[i];
    u64 v = 1;
    for (u64 s : src) v = mul_mod(v, s, p);
    (*inv)[i] = to_mont(inv_mod(v, p), p);
  }
  if (!pad) return;
  const int rl = re - rs;
  pad->assign(dl - rl, 0);
  for (int i = 0; i < static_cast<int>(dl) - rl; i++) {
    const int pi = i >= rs ? i + rl : i;
    const u64 p = dst[pi];
    u64 v = 1;
    for (int j = rs; j < re; j++) v = mul_mod(v, dst[j], p);
    (*pad)[i] = to_mont(v, p);
  }
}
i64 *upload(const std::vector<i64> &v) {
  i64 *p = nullptr;
  if (v.empty()) return nullptr;
  if (cudaMalloc(&p, v.size() * 8) != cudaSuccess) return nullptr;
  cudaMemcpy(p, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
  return p;
}
}  // namespace

void build_level_ms64(const Params64 &P, int level, LevelMS64 *out) {
  // ModSwitch.cu:175-318 (levels 0 .. max; the 64-bit path has no
  // sparse-secret level -1)
  LevelMS64 &m = *out;
  const u64 n = static_cast<u64>(P.n);
  m.level = level;
  m.num_aux = P.alpha;
  NP np = P.level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  m.num_q = nq;
  m.beta = (np.main + P.max_ter + m.num_aux - 1) / m.num_aux;
  std::vector<int> g(tot);
  P.gidx(np, g.data());
  std::vector<u64> lp(tot);
  for (int i = 0; i < tot; i++) lp[i] = P.primes[g[i]];
  const int padded = np.main + P.max_ter;
  const int npad = padded - nq;
  m.mod_up1.assign(nq, 0);
  m.dig_s.assign(m.beta, 0);
  m.dig_e.assign(m.beta, 0);
  m.mod_up2.assign(m.beta, {});
  for (int i = 0; i < m.beta; i++) {
    int s = i * m.num_aux, e = std::min((i + 1) * m.num_aux, padded);
    if (e <= npad) continue;
    s = std::max(0, s - npad);
    e -= npad;
    m.dig_s[i] = s;
    m.dig_e[i] = e;
    std::vector<u64> src(lp.begin() + s, lp.begin() + e), dst(lp.begin(), lp.begin() + s);
    dst.insert(dst.end(), lp.begin() + e, lp.end());
    std::vector<u64> c1;
    ms_consts(n, src, dst, 0, 0, &c1, &m.mod_up2[i]);
    std::copy(c1.begin(), c1.end(), m.mod_up1.begin() + s);
  }
  std::vector<u64> qp(lp.begin(), lp.begin() + nq), pp(lp.begin() + nq, lp.end());
  ms_consts(n, pp, qp, 0, 0, &m.mod_down1, &m.mod_down2);
  epi_consts(pp, qp, 0, 0, &m.inv_p_prod, nullptr);
  if (level <= 0) return;
  NP nn = P.level_np(level - 1, m.num_aux);
  std::vector<int> gn(nn.total());
  P.gidx(nn, gn.data());
  const int nnq = nn.q();
  std::vector<u64> next(nnq);
  for (int i = 0; i < nnq; i++) next[i] = P.primes[gn[i]];
  const int md = np.main - nn.main, td = np.ter - nn.ter;
  std::vector<u64> rs_src;
  if (td > 0) {
    if (md > 0) return;
    rs_src.assign(lp.begin(), lp.begin() + td);
    m.restore_start = nnq + md;
    m.restore_end = nnq;
  } else if (md > 0) {
    rs_src.assign(lp.begin() + nq - md, lp.begin() + nq);
    m.restore_start = 0;
    m.restore_end = -td;
  } else {
    return;
  }
  m.has_rescale = true;
  std::vector<u64> mdr_src = rs_src;
  mdr_src.insert(mdr_src.end(), pp.begin(), pp.end());
  ms_consts(n, rs_src, next, m.restore_start, m.restore_end, &m.rs1, &m.rs2);
  epi_consts(rs_src, next, m.restore_start, m.restore_end, &m.rs_inv, &m.rs_pad);
  ms_consts(n, mdr_src, next, m.restore_start, m.restore_end, &m.mdr1, &m.mdr2);
  epi_consts(mdr_src, next, m.restore_start, m.restore_end, &m.mdr_inv, &m.mdr_pad);
}

// ------------------------------------------------------------ objects
Ct64::~Ct64() {
  cudaFree(bx);
  cudaFree(ax);
  cudaFree(rx);
}

Status Ct64::reserve(const NP &want, int n, bool with_rx) {
  const size_t words = static_cast<size_t>(want.total()) * n;
  if (words > cap_words) {
    cudaFree(bx);
    cudaFree(ax);
    bx = ax = nullptr;
    cap_words = 0;
    if (cudaMalloc(&bx, words * 8) != cudaSuccess || cudaMalloc(&ax, words * 8) != cudaSuccess) {
      set_error("ciphertext allocation failed");
      return kErrAlloc;
    }
    cap_words = words;
  }
  if (with_rx && words > rx_cap_words) {
    cudaFree(rx);
    rx = nullptr;
    rx_cap_words = 0;
    if (cudaMalloc(&rx, words * 8) != cudaSuccess) {
      set_error("ciphertext allocation failed");
      return kErrAlloc;
    }
    rx_cap_words = words;
  }
  np = want;
  has_rx = with_rx;
  return kOk;
}

void Ct64::swap(Ct64 &o) {
  std::swap(np, o.np);
  std::swap(scale, o.scale);
  std::swap(num_slots, o.num_slots);
  std::swap(has_rx, o.has_rx);
  std::swap(bx, o.bx);
  std::swap(ax, o.ax);
  std::swap(rx, o.rx);
  std::swap(cap_words, o.cap_words);
  std::swap(rx_cap_words, o.rx_cap_words);
}

Evk64::~Evk64() {
  cudaFree(bx);
  cudaFree(ax);
}

Context64::~Context64() {
  if (P) cudaSetDevice(device);
  for (auto &m : ms)
    if (m) {
      for (auto *t : m->d_mod_up2) cudaFree(t);
      cudaFree(m->d_mod_down2);
      cudaFree(m->d_rs2);
      cudaFree(m->d_mdr2);
    }
  cudaFree(d_primes);
  cudaFree(d_qinv);
  cudaFree(d_tw);
  cudaFree(d_itw);
  if (stream && own_stream) cudaStreamDestroy(stream);
}

Status Context64::check(const char *where) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

void Context64::shoup(u64 c, int g, u64 *w, u64 *ws) const {
  const u64 q = P->primes[g];
  *w = c % q;
  *ws = static_cast<u64>((static_cast<u128>(*w) << 64) / q);
}

void Context64::mont_shoup(u64 c, int g, u64 *w, u64 *ws) const { shoup(mul_mod(c, r_inv[g], P->primes[g]), g, w, ws); }

Status Context64::init(const ParamSpec64 &spec, int dev, std::string *err) {
  P = Params64::create(spec, err);
  if (!P) return kErrInvalidArg;
  device = dev;
  if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    *err = "device or stream setup failed";
    return kErrCuda;
  }
  const int n = P->n, np_all = P->L + P->alpha;
  // twiddles (NTT.cu:1233-1299, word = uint64_t): psi_rev[j] = psi^brev(j),
  // stored plain with the Shoup companion floor(w 2^64 / q)
  std::vector<ulonglong2> tw(static_cast<size_t>(np_all) * n), itw(tw.size());
  n_inv.resize(np_all);
  n_inv_mont_inv.resize(np_all);
  mont_conv.resize(np_all);
  r_inv.resize(np_all);
  std::vector<u64> pw(n), pwi(n);
  for (int g = 0; g < np_all; g++) {
    const u64 q = P->primes[g];
    const u64 psi = primitive_root(2ull * n, q), psi_inv = inv_mod(psi, q);
    n_inv[g] = inv_mod(static_cast<u64>(n), q);
    n_inv_mont_inv[g] = to_mont(n_inv[g], q);
    mont_conv[g] = to_mont(to_mont(1, q), q);
    r_inv[g] = inv_mod(to_mont(1, q), q);
    pw[0] = pwi[0] = 1;
    for (int j = 1; j < n; j++) {
      pw[j] = mul_mod(pw[j - 1], psi, q);
      pwi[j] = mul_mod(pwi[j - 1], psi_inv, q);
    }
    imag_unit.push_back(to_mont(pw[n / 2], q));  // psi^(N/2) = psi_rev[1]
    for (int j = 0; j < n; j++) {
      const unsigned r = brev(j, P->log_n);
      auto sh = [q](u64 w) { return static_cast<u64>((static_cast<u128>(w) << 64) / q); };
      tw[static_cast<size_t>(g) * n + j] = make_ulonglong2(pw[r], sh(pw[r]));
      itw[static_cast<size_t>(g) * n + j] = make_ulonglong2(pwi[r], sh(pwi[r]));
    }
  }
  if (cudaMalloc(&d_primes, np_all * 8) != cudaSuccess || cudaMalloc(&d_qinv, np_all * 8) != cudaSuccess ||
      cudaMalloc(&d_tw, tw.size() * sizeof(ulonglong2)) != cudaSuccess ||
      cudaMalloc(&d_itw, itw.size() * sizeof(ulonglong2)) != cudaSuccess) {
    *err = "device allocation failed";
    return kErrAlloc;
  }
  cudaMemcpy(d_primes, P->primes.data(), np_all * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_qinv, P->qinv.data(), np_all * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice);
  cudaMemcpy(d_itw, itw.data(), itw.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice);
  // P mod q_i (Montgomery), Context.cpp:78-90
  p_prod.resize(P->L);
  for (int i = 0; i < P->L; i++) {
    const u64 q = P->primes[i];
    u64 v = 1;
    for (int a = 0; a < P->alpha; a++) v = mul_mod(v, P->primes[P->L + a], q);
    p_prod[i] = to_mont(v, q);
  }
  ms.resize(P->max_level + 2);
  return check("context64 init");
}

const LevelMS64 &Context64::lms(int level) {
  auto &slot = ms.at(level + 1);
  if (!slot) {
    slot = std::make_unique<LevelMS64>();
    build_level_ms64(*P, level, slot.get());
    for (auto &t : slot->mod_up2) slot->d_mod_up2.push_back(t.empty() ? nullptr : upload(t));
    slot->d_mod_down2 = upload(slot->mod_down2);
    slot->d_rs2 = upload(slot->rs2);
    slot->d_mdr2 = upload(slot->mdr2);
  }
  return *slot;
}

namespace {
template <typename F>
void for_batches64(const std::vector<Row64> &rows, F &&launch) {
  RowBatch64 rb;
  rb.count = 0;
  for (const Row64 &r : rows) {
    rb.rows[rb.count++] = r;
    if (rb.count == kMaxRows64) {
      launch(rb);
      rb.count = 0;
    }
  }
  if (rb.count) launch(rb);
}
}  // namespace

Status Context64::ntt(const NP &np, u64 *data, int count, bool mont) {
  // NTTHandler::NTT (NTT.cu:606-671): optional conversion to Montgomery form
  const int tot = np.total(), n = P->n;
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  std::vector<Row64> rows;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < tot; i++) {
      Row64 r{};
      r.src = r.dst = data + (static_cast<size_t>(c) * tot + i) * n;
      r.tw = tw(g[i]);
      r.q = P->primes[g[i]];
      mont_shoup(mont_conv[g[i]], g[i], &r.c0, &r.c0s);
      r.flags = mont ? kPreMult : 0u;
      rows.push_back(r);
    }
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_fwd(rb, stream); });
  return check("ntt64");
}

Status Context64::intt(const NP &np, u64 *data, int count, bool mont) {
  // NTTHandler::INTT (NTT.cu:673-741)
  const int tot = np.total(), n = P->n;
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  std::vector<Row64> rows;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < tot; i++) {
      Row64 r{};
      r.src = r.dst = data + (static_cast<size_t>(c) * tot + i) * n;
      r.tw = itw(g[i]);
      r.q = P->primes[g[i]];
      mont_shoup(mont ? n_inv[g[i]] : n_inv_mont_inv[g[i]], g[i], &r.c0, &r.c0s);
      rows.push_back(r);
    }
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_inv(rb, stream); });
  return check("intt64");
}

Status Context64::modup(int level, const u64 *src, u64 *dst) {
  // ModSwitchHandler::ModUp (ModSwitch.cu:429-509): INTT of the q limbs times
  // the digit constants (centred), per digit a copy of its own limbs, the
  // base conversion to the other primes and their NTT
  const LevelMS64 &m = lms(level);
  const int n = P->n;
  const NP np = P->level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  ArenaScope scope(arena);
  i64 *xt = static_cast<i64 *>(arena.alloc(static_cast<size_t>(nq) * n * 8));
  if (!xt) {
    set_error("modup64: scratch allocation failed");
    return kErrAlloc;
  }
  std::vector<Row64> rows;
  for (int r = 0; r < nq; r++) {
    Row64 d{};
    d.src = src + static_cast<size_t>(r) * n;
    d.dst = reinterpret_cast<u64 *>(xt) + static_cast<size_t>(r) * n;
    d.tw = itw(g[r]);
    d.q = P->primes[g[r]];
    mont_shoup(m.mod_up1[r], g[r], &d.c0, &d.c0s);
    d.flags = kCentre;
    rows.push_back(d);
  }
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_inv(rb, stream); });
  BConv64Batch b{};
  b.primes = d_primes;
  b.qinvs = d_qinv;
  const size_t out_words = static_cast<size_t>(tot) * n;
  rows.clear();
  for (int i = 0; i < m.beta; i++) {
    const int s = m.dig_s[i], e = m.dig_e[i];
    if (e <= 0) continue;
    u64 *out = dst + i * out_words;
    cudaMemcpyAsync(out + static_cast<size_t>(s) * n, src + static_cast<size_t>(s) * n,
                    static_cast<size_t>(e - s) * n * 8, cudaMemcpyDeviceToDevice, stream);
    BConv64Job &j = b.jobs[b.count++];
    j.xt = xt + static_cast<size_t>(s) * n;
    j.out = out;
    j.table = m.d_mod_up2[i];
    j.K = e - s;
    j.M = tot - (e - s);
    int k = 0;
    for (int r = 0; r < tot; r++) {
      if (r >= s && r < e) continue;
      j.out_row[k] = static_cast<uint8_t>(r);
      j.out_gidx[k] = static_cast<uint8_t>(g[r]);
      k++;
      Row64 d{};
      d.src = d.dst = out + static_cast<size_t>(r) * n;
      d.tw = tw(g[r]);
      d.q = P->primes[g[r]];
      rows.push_back(d);
    }
    if (b.count == kMaxBConv64Jobs) {
      launch_bconv64(b, stream);
      b.count = 0;
    }
  }
  launch_bconv64(b, stream);
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_fwd(rb, stream); });
  return check("modup64");
}

Status Context64::moddown(int level, MDType type, const u64 *const *src, u64 *const *dst, int npoly) {
  // ModSwitch.cu:566-684 with the NTT epilogue of NTT.cu:456-601 (word =
  // uint64_t)
  const LevelMS64 &m = lms(level);
  const int n = P->n;
  CHD_CHECK(type == MDType::kModDown || m.has_rescale, kErrInvalidLevel, "rescale not available at this level");
  const int nsa = type == MDType::kRescale ? 0 : m.num_aux;
  NP ns = P->level_np(level, nsa);
  NP nd = P->level_np(type == MDType::kModDown ? level : level - 1, 0);
  NP nn{std::min(ns.main, nd.main), std::min(ns.ter, nd.ter), 0};
  const int src_len = ns.total() - nn.total(), dst_len = nd.total();
  CHD_CHECK(src_len >= 1 && src_len <= 16 && dst_len <= 64, kErrUnsupported, "moddown64: shape out of range");
  const u64 *c1 = type == MDType::kModDown ? m.mod_down1.data()
                  : type == MDType::kRescale ? m.rs1.data() : m.mdr1.data();
  const i64 *table = type == MDType::kModDown ? m.d_mod_down2 : type == MDType::kRescale ? m.d_rs2 : m.d_mdr2;
  const u64 *inv = type == MDType::kModDown ? m.inv_p_prod.data()
                   : type == MDType::kRescale ? m.rs_inv.data() : m.mdr_inv.data();
  const u64 *pad = type == MDType::kModDown ? nullptr : type == MDType::kRescale ? m.rs_pad.data() : m.mdr_pad.data();
  std::vector<int> gs(ns.total()), gd(nd.total());
  P->gidx(ns, gs.data());
  P->gidx(nd, gd.data());
  std::vector<int> srows;
  const bool on_main = ns.main > nn.main, on_ter = ns.ter > nn.ter;
  CHD_CHECK(!(on_main && on_ter), kErrInvalidArg, "moddown64: invalid prime combination");
  if (!on_ter)
    for (int r = ns.ter + nn.main; r < ns.q(); r++) srows.push_back(r);
  else
    for (int r = 0; r < ns.ter - nn.ter; r++) srows.push_back(r);
  for (int a = 0; a < nsa; a++) srows.push_back(ns.q() + a);
  CHD_CHECK(static_cast<int>(srows.size()) == src_len, kErrInvalidArg, "moddown64: internal row mismatch");
  ArenaScope scope(arena);
  i64 *xt = static_cast<i64 *>(arena.alloc(static_cast<size_t>(npoly) * src_len * n * 8));
  if (!xt) {
    set_error("moddown64: scratch allocation failed");
    return kErrAlloc;
  }
  std::vector<Row64> rows;
  for (int p = 0; p < npoly; p++)
    for (int i = 0; i < src_len; i++) {
      const int gg = gs[srows[i]];
      Row64 d{};
      d.src = src[p] + static_cast<size_t>(srows[i]) * n;
      d.dst = reinterpret_cast<u64 *>(xt) + (static_cast<size_t>(p) * src_len + i) * n;
      d.tw = itw(gg);
      d.q = P->primes[gg];
      mont_shoup(c1[i], gg, &d.c0, &d.c0s);
      d.flags = kCentre;
      rows.push_back(d);
    }
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_inv(rb, stream); });
  BConv64Batch b{};
  b.primes = d_primes;
  b.qinvs = d_qinv;
  for (int p = 0; p < npoly; p++) {
    BConv64Job &j = b.jobs[b.count++];
    j.xt = xt + static_cast<size_t>(p) * src_len * n;
    j.out = dst[p];
    j.table = table;
    j.K = src_len;
    j.M = dst_len;
    for (int y = 0; y < dst_len; y++) {
      j.out_row[y] = static_cast<uint8_t>(y);
      j.out_gidx[y] = static_cast<uint8_t>(gd[y]);
    }
    if (b.count == kMaxBConv64Jobs) {
      launch_bconv64(b, stream);
      b.count = 0;
    }
  }
  launch_bconv64(b, stream);
  const int src2_start = nd.ter - nn.ter, src2_end = src2_start + nn.q();
  const int src2_off = std::max(0, ns.ter - nd.ter);
  rows.clear();
  for (int p = 0; p < npoly; p++)
    for (int y = 0; y < dst_len; y++) {
      Row64 d{};
      d.src = d.dst = dst[p] + static_cast<size_t>(y) * n;
      d.tw = tw(gd[y]);
      d.q = P->primes[gd[y]];
      mont_shoup(inv[y], gd[y], &d.c2, &d.c2s);
      d.flags = kModDownEpi;
      if (y >= src2_start && y < src2_end) {
        d.flags |= kHasSrc2;
        d.src2 = src[p] + static_cast<size_t>(src2_off + y - src2_start) * n;
        if (pad) {
          d.flags |= kPadSrc2;
          mont_shoup(pad[y - src2_start], gd[y], &d.c1, &d.c1s);
        }
      }
      rows.push_back(d);
    }
  for_batches64(rows, [&](const RowBatch64 &rb) { launch_ntt64_fwd(rb, stream); });
  return check("moddown64");
}

Status Context64::key_mult(int level, const u64 *d, const u64 *d0, const u64 *d1, const Evk64 &key, u64 *acc_b,
                           u64 *acc_a) {
  // MultKeyNoModDown (Context.cpp:609-648): ModUp of d, then the inner
  // product with the key's digits over Q u P, plus P (d0, d1) on the q rows
  // (the CAccum of Context.cpp:687-699)
  const LevelMS64 &m = lms(level);
  const int n = P->n;
  const NP np = P->level_np(level, P->alpha);
  const int nq = np.q(), tot = np.total();
  CHD_CHECK(key.np.aux == P->alpha && key.np.q() == P->L, kErrKey, "key switch: key basis mismatch");
  CHD_CHECK(m.beta <= 8, kErrUnsupported, "key switch: more than 8 digits");
  const size_t mw = static_cast<size_t>(tot) * n;
  ArenaScope scope(arena);
  u64 *mu = static_cast<u64 *>(arena.alloc(m.beta * mw * 8));
  if (!mu) {
    set_error("key switch: scratch allocation failed");
    return kErrAlloc;
  }
  CHD_TRY(modup(level, d, mu));
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  const int prime_offset = P->max_ter - np.ter;
  const size_t kstride = static_cast<size_t>(key.np.total()) * n;
  KeyMac64Batch kb{};
  for (int r = 0; r < tot; r++) {
    KeyMac64Row &row = kb.rows[kb.count++];
    row = KeyMac64Row{};
    const int key_row = r < nq ? prime_offset + r : P->L + (r - nq);
    int nb = 0;
    for (int i = 0; i < m.beta; i++) {
      if (m.dig_e[i] <= 0) continue;
      CHD_CHECK(i < key.beta, kErrKey, "key switch: key has too few digits");
      row.mu[nb] = mu + i * mw + static_cast<size_t>(r) * n;
      row.kb[nb] = key.bx + i * kstride + static_cast<size_t>(key_row) * n;
      row.ka[nb] = key.ax + i * kstride + static_cast<size_t>(key_row) * n;
      nb++;
    }
    row.beta = nb;
    row.acc_b = acc_b + static_cast<size_t>(r) * n;
    row.acc_a = acc_a + static_cast<size_t>(r) * n;
    row.q = P->primes[g[r]];
    row.qinv = P->qinv[g[r]];
    row.p = r < nq ? p_prod[prime_offset + r] : 0;
    row.d0 = r < nq && d0 ? d0 + static_cast<size_t>(r) * n : nullptr;
    row.d1 = r < nq && d1 ? d1 + static_cast<size_t>(r) * n : nullptr;
    if (kb.count == kMaxKeyMac64Rows) {
      launch_key_mac64(kb, stream);
      kb.count = 0;
    }
  }
  launch_key_mac64(kb, stream);
  return check("key switch64");
}

namespace {
int level_of(const Params64 &P, const Ct64 &a) { return P.np_to_level(NP{a.np.main, a.np.ter, 0}); }
}  // namespace

Status Context64::hmult(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key, bool do_rescale) {
  // Context::HMult (Context.cpp:862-871): tensor, then the key switch of d2
  // with P (d0, d1) added, then ModDown or the merged ModDownAndRescale
  CHD_CHECK(a.np == b.np && a.np.aux == 0, kErrShape, "HMult: operands must share a level and have no aux primes");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "HMult: invalid level");
  CHD_CHECK(!do_rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  const int n = P->n, nq = a.np.q(), tot = nq + P->alpha;
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  const size_t qw = static_cast<size_t>(nq) * n, tw_ = static_cast<size_t>(tot) * n;
  ArenaScope scope(arena);
  u64 *d = static_cast<u64 *>(arena.alloc(3 * qw * 8));
  u64 *acc = static_cast<u64 *>(arena.alloc(2 * tw_ * 8));
  if (!d || !acc) {
    set_error("HMult: scratch allocation failed");
    return kErrAlloc;
  }
  Elem64Batch eb{};
  for (int r = 0; r < nq; r++) {
    Elem64Row &e = eb.rows[eb.count++];
    const size_t o = static_cast<size_t>(r) * n;
    e.b1 = a.bx + o;
    e.a1 = a.ax + o;
    e.b2 = b.bx + o;
    e.a2 = b.ax + o;
    e.o0 = d + o;
    e.o1 = d + qw + o;
    e.o2 = d + 2 * qw + o;
    e.q = P->primes[g[r]];
    e.qinv = P->qinv[g[r]];
    if (eb.count == kMaxElem64Rows) {
      launch_tensor64(eb, stream);
      eb.count = 0;
    }
  }
  launch_tensor64(eb, stream);
  u64 *acc_b = acc, *acc_a = acc + tw_;
  CHD_TRY(key_mult(level, d + 2 * qw, d, d + qw, key, acc_b, acc_a));
  const NP out_np = P->level_np(do_rescale ? level - 1 : level, 0);
  const double sc = do_rescale ? a.scale * b.scale / P->rescale_prod[level] : a.scale * b.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  CHD_TRY(res.reserve(out_np, n));
  const u64 *srcs[2] = {acc_b, acc_a};
  u64 *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, do_rescale ? MDType::kModDownRescale : MDType::kModDown, srcs, dsts, 2));
  res.scale = sc;
  res.num_slots = slots;
  return check("hmult64");
}

Status Context64::hrot(Ct64 &res, const Ct64 &a, const Evk64 &key, int dist) {
  // Context::HRot (Context.cpp:776-791): MultKey, then the automorphism
  const int slots = a.num_slots > 0 ? a.num_slots : P->n / 2;
  dist %= slots;
  if (dist < 0) dist += slots;
  return key_switch_permute(res, a, key, P->galois_of(dist));
}

Status Context64::hconj(Ct64 &res, const Ct64 &a, const Evk64 &key) {
  // Context::HConj (Context.cpp:793-798): MultKey, then the conjugation
  return key_switch_permute(res, a, key, P->galois_of(-1));
}

Status Context64::key_switch_permute(Ct64 &res, const Ct64 &a, const Evk64 &key, u64 galois) {
  CHD_CHECK(a.np.aux == 0, kErrShape, "HRot: no aux primes");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "HRot: invalid level");
  CHD_CHECK(&res != &a, kErrInvalidArg, "HRot64: the result must not alias the input");
  const int n = P->n, nq = a.np.q(), tot = nq + P->alpha;
  const size_t qw = static_cast<size_t>(nq) * n, tw_ = static_cast<size_t>(tot) * n;
  ArenaScope scope(arena);
  u64 *acc = static_cast<u64 *>(arena.alloc(2 * tw_ * 8));
  u64 *ks = static_cast<u64 *>(arena.alloc(2 * qw * 8));
  if (!acc || !ks) {
    set_error("HRot: scratch allocation failed");
    return kErrAlloc;
  }
  u64 *acc_b = acc, *acc_a = acc + tw_;
  // MultKey (Context.cpp:584-607): d_in = ax, d0 = bx
  CHD_TRY(key_mult(level, a.ax, a.bx, nullptr, key, acc_b, acc_a));
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  const u64 *srcs[2] = {acc_b, acc_a};
  u64 *dsts[2] = {ks, ks + qw};
  CHD_TRY(moddown(level, MDType::kModDown, srcs, dsts, 2));
  const double sc = a.scale;
  const int sl = a.num_slots;
  const NP np = a.np;
  CHD_TRY(res.reserve(np, n));
  Elem64Batch eb{};
  for (int p = 0; p < 2; p++)
    for (int r = 0; r < nq; r++) {
      Elem64Row &e = eb.rows[eb.count++];
      e = Elem64Row{};
      e.a1 = ks + p * qw + static_cast<size_t>(r) * n;
      e.o0 = (p == 0 ? res.bx : res.ax) + static_cast<size_t>(r) * n;
      e.q = P->primes[g[r]];
      if (eb.count == kMaxElem64Rows) {
        launch_permute64(eb, galois, stream);
        eb.count = 0;
      }
    }
  launch_permute64(eb, galois, stream);
  res.scale = sc;
  res.num_slots = sl;
  return check("hrot64");
}

Status Context64::rescale(Ct64 &res, const Ct64 &a) {
  // Context::Rescale (Context.cpp:739-774)
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  CHD_CHECK(&res != &a, kErrInvalidArg, "Rescale64: the result must not alias the input");
  CHD_TRY(res.reserve(P->level_np(level - 1), P->n));
  const u64 *srcs[2] = {a.bx, a.ax};
  u64 *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, MDType::kRescale, srcs, dsts, 2));
  res.scale = a.scale / P->rescale_prod[level];
  res.num_slots = a.num_slots;
  return kOk;
}

// ---- Context<uint64_t> operations (Context.cpp:101-949) ----------------

namespace {
// round-toward-zero integer of v reduced to [0, p), exact for every finite
// double (|v| >= 2^53 is an integer m 2^e)
u64 trunc_mod64(double v, u64 p) {
  if (v == 0.0) return 0;
  const bool neg = v < 0;
  const double a = std::fabs(v);
  u64 r;
  if (a < 18446744073709551616.0) {
    r = static_cast<u64>(a) % p;
  } else {
    int e;
    const double m = std::frexp(a, &e);
    const u64 mi = static_cast<u64>(std::ldexp(m, 53));
    r = mul_mod(mi % p, pow_mod(2, e - 53, p), p);
  }
  if (neg && r) r = p - r;
  return r;
}
}  // namespace

void Context64::encode_const(int level, double scale, double value, int num_aux, std::vector<u64> *cx) const {
  const NP np = P->level_np(level, num_aux);
  std::vector<int> g(np.total());
  P->gidx(np, g.data());
  cx->resize(np.total());
  const double v = value * scale;
  for (int k = 0; k < np.total(); k++) (*cx)[k] = to_mont(trunc_mod64(v, P->primes[g[k]]), P->primes[g[k]]);
}

namespace {
// one element-wise op over `parts` parts of every row of np
Status elem_parts64(Context64 &C, Elem64Op op, const NP &np, int parts, u64 *const *dst, const u64 *const *a,
                    const u64 *const *b, const u64 *k) {
  const int n = C.P->n, tot = np.total();
  std::vector<int> g(tot);
  C.P->gidx(np, g.data());
  Elem64Batch eb{};
  for (int p = 0; p < parts; p++)
    for (int r = 0; r < tot; r++) {
      Elem64Row &e = eb.rows[eb.count++];
      e = Elem64Row{};
      const size_t o = static_cast<size_t>(r) * n;
      e.a1 = a[p] + o;
      e.b1 = b ? b[p] + o : nullptr;
      e.o0 = dst[p] + o;
      e.q = C.P->primes[g[r]];
      e.qinv = C.P->qinv[g[r]];
      e.c = k ? k[r] : 0;
      if (eb.count == kMaxElem64Rows) {
        launch_elem64(op, eb, C.stream);
        eb.count = 0;
      }
    }
  launch_elem64(op, eb, C.stream);
  return C.check("elementwise64");
}

// the result of an operation that grows `res` while res is also an operand:
// compute into a temporary, then take its buffers
template <class F>
Status via_temp(Ct64 &res, F &&f) {
  Ct64 tmp;
  CHD_TRY(f(tmp));
  res.swap(tmp);
  return kOk;
}
}  // namespace

Status Context64::copy(Ct64 &res, const Ct64 &a) {
  if (&res == &a) return kOk;
  const NP np = a.np;
  CHD_TRY(res.reserve(np, P->n, a.has_rx));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 8;
  cudaMemcpyAsync(res.bx, a.bx, bytes, cudaMemcpyDeviceToDevice, stream);
  cudaMemcpyAsync(res.ax, a.ax, bytes, cudaMemcpyDeviceToDevice, stream);
  if (a.has_rx) cudaMemcpyAsync(res.rx, a.rx, bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = a.scale;
  res.num_slots = a.num_slots;
  return check("copy64");
}

Status Context64::add(Ct64 &res, const Ct64 &a, const Ct64 &b) {
  // Context.cpp:145-172: with rx on one side only, the result keeps it
  CHD_CHECK(a.np == b.np, kErrShape, "Add: level mismatch");
  const bool out_rx = a.has_rx || b.has_rx, both_rx = a.has_rx && b.has_rx;
  if ((&res == &a || &res == &b) && out_rx && !res.has_rx)
    return via_temp(res, [&](Ct64 &t) { return add(t, a, b); });
  const u64 *keep_rx = (!both_rx && out_rx) ? (a.has_rx ? a.rx : b.rx) : nullptr;
  const NP np = a.np;
  const u64 *pa[3] = {a.bx, a.ax, a.rx}, *pb[3] = {b.bx, b.ax, b.rx};
  const double sc = a.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  CHD_TRY(res.reserve(np, P->n, out_rx));
  u64 *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kAdd, np, both_rx ? 3 : 2, pd, pa, pb, nullptr));
  if (keep_rx && keep_rx != res.rx)
    cudaMemcpyAsync(res.rx, keep_rx, static_cast<size_t>(np.total()) * P->n * 8, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return check("add64");
}

Status Context64::sub(Ct64 &res, const Ct64 &a, const Ct64 &b) {
  // Context.cpp:205-229: with rx on one side only, res.rx = a.rx or -b.rx
  CHD_CHECK(a.np == b.np, kErrShape, "Sub: level mismatch");
  const bool out_rx = a.has_rx || b.has_rx, both_rx = a.has_rx && b.has_rx;
  if ((&res == &a || &res == &b) && out_rx && !res.has_rx)
    return via_temp(res, [&](Ct64 &t) { return sub(t, a, b); });
  const u64 *only_rx = (!both_rx && out_rx) ? (a.has_rx ? a.rx : b.rx) : nullptr;
  const bool neg_rx = !both_rx && b.has_rx;
  const NP np = a.np;
  const u64 *pa[3] = {a.bx, a.ax, a.rx}, *pb[3] = {b.bx, b.ax, b.rx};
  const double sc = a.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  CHD_TRY(res.reserve(np, P->n, out_rx));
  u64 *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kSub, np, both_rx ? 3 : 2, pd, pa, pb, nullptr));
  if (neg_rx) {
    const u64 *src[1] = {only_rx};
    u64 *dst[1] = {res.rx};
    CHD_TRY(elem_parts64(*this, Elem64Op::kNeg, np, 1, dst, src, nullptr, nullptr));
  } else if (only_rx && only_rx != res.rx) {
    cudaMemcpyAsync(res.rx, only_rx, static_cast<size_t>(np.total()) * P->n * 8, cudaMemcpyDeviceToDevice, stream);
  }
  res.scale = sc;
  res.num_slots = slots;
  return check("sub64");
}

Status Context64::neg(Ct64 &res, const Ct64 &a) {
  const NP np = a.np;
  const bool rx = a.has_rx;
  const u64 *pa[3] = {a.bx, a.ax, a.rx};
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, P->n, rx));
  u64 *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kNeg, np, rx ? 3 : 2, pd, pa, nullptr, nullptr));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context64::mult_tensor(Ct64 &res, const Ct64 &a, const Ct64 &b) {
  // Context.cpp:316-330: (b1 b2, b1 a2 + a1 b2, a1 a2)
  CHD_CHECK(a.np == b.np && a.np.aux == 0, kErrShape, "Mult: level mismatch");
  CHD_CHECK(!a.has_rx && !b.has_rx, kErrShape, "Relinearization required before Mult Ct x Ct");
  CHD_CHECK(&res != &a && &res != &b, kErrInvalidArg, "Mult: result must not alias an operand");
  const int n = P->n, nq = a.np.q();
  CHD_TRY(res.reserve(a.np, n, true));
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  Elem64Batch eb{};
  for (int r = 0; r < nq; r++) {
    Elem64Row &e = eb.rows[eb.count++];
    e = Elem64Row{};
    const size_t o = static_cast<size_t>(r) * n;
    e.b1 = a.bx + o;
    e.a1 = a.ax + o;
    e.b2 = b.bx + o;
    e.a2 = b.ax + o;
    e.o0 = res.bx + o;
    e.o1 = res.ax + o;
    e.o2 = res.rx + o;
    e.q = P->primes[g[r]];
    e.qinv = P->qinv[g[r]];
    if (eb.count == kMaxElem64Rows) {
      launch_tensor64(eb, stream);
      eb.count = 0;
    }
  }
  launch_tensor64(eb, stream);
  res.scale = a.scale * b.scale;
  res.num_slots = std::max(a.num_slots, b.num_slots);
  return check("mult64");
}

Status Context64::relinearize(Ct64 &res, const Ct64 &a, const Evk64 &key, bool do_rescale) {
  // Relinearize / RelinearizeRescale (Context.cpp:650-737): the key switch
  // of rx with P (bx, ax) added, then ModDown or ModDownAndRescale
  CHD_CHECK(a.has_rx && a.np.aux == 0, kErrShape, "Relinearize: input must have rx and no aux primes");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "Relinearize: invalid level");
  CHD_CHECK(!do_rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  if (&res == &a) return via_temp(res, [&](Ct64 &t) { return relinearize(t, a, key, do_rescale); });
  const int n = P->n, tot = a.np.q() + P->alpha;
  const size_t tw_ = static_cast<size_t>(tot) * n;
  ArenaScope scope(arena);
  u64 *acc = static_cast<u64 *>(arena.alloc(2 * tw_ * 8));
  if (!acc) {
    set_error("Relinearize: scratch allocation failed");
    return kErrAlloc;
  }
  CHD_TRY(key_mult(level, a.rx, a.bx, a.ax, key, acc, acc + tw_));
  const double sc = do_rescale ? a.scale / P->rescale_prod[level] : a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(P->level_np(do_rescale ? level - 1 : level), n));
  const u64 *srcs[2] = {acc, acc + tw_};
  u64 *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, do_rescale ? MDType::kModDownRescale : MDType::kModDown, srcs, dsts, 2));
  res.scale = sc;
  res.num_slots = slots;
  return check("relinearize64");
}

Status Context64::mult_key(Ct64 &res, const Ct64 &a, const Evk64 &key) {
  // MultKey (Context.cpp:584-607): the key switch of ax, P bx added to the
  // b accumulator, then ModDown
  CHD_CHECK(!a.has_rx && a.np.aux == 0, kErrShape, "MultKey: input must be relinearised, without aux primes");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "MultKey: invalid level");
  if (&res == &a) return via_temp(res, [&](Ct64 &t) { return mult_key(t, a, key); });
  const int n = P->n, tot = a.np.q() + P->alpha;
  const size_t tw_ = static_cast<size_t>(tot) * n;
  ArenaScope scope(arena);
  u64 *acc = static_cast<u64 *>(arena.alloc(2 * tw_ * 8));
  if (!acc) {
    set_error("MultKey: scratch allocation failed");
    return kErrAlloc;
  }
  CHD_TRY(key_mult(level, a.ax, a.bx, nullptr, key, acc, acc + tw_));
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(a.np, n));
  const u64 *srcs[2] = {acc, acc + tw_};
  u64 *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, MDType::kModDown, srcs, dsts, 2));
  res.scale = sc;
  res.num_slots = slots;
  return check("mult_key64");
}

Status Context64::permute(Ct64 &res, const Ct64 &a, int rot, bool conjugate) {
  // Permute / PermuteConjugate (Context.cpp:486-530): the automorphism on
  // every part
  CHD_CHECK(a.np.aux == 0, kErrShape, "Permute: no aux primes");
  u64 galois = 0;
  if (conjugate) {
    galois = P->galois_of(-1);
  } else {
    const int slots = a.num_slots > 0 ? a.num_slots : P->n / 2;
    int amount = rot % slots;
    if (amount < 0) amount += slots;
    if (amount == 0) return copy(res, a);
    galois = P->galois_of(amount);
  }
  if (&res == &a) return via_temp(res, [&](Ct64 &t) { return permute(t, a, rot, conjugate); });
  const int n = P->n, nq = a.np.q();
  const bool rx = a.has_rx;
  CHD_TRY(res.reserve(a.np, n, rx));
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  const u64 *src[3] = {a.bx, a.ax, a.rx};
  u64 *dst[3] = {res.bx, res.ax, res.rx};
  Elem64Batch eb{};
  for (int p = 0; p < (rx ? 3 : 2); p++)
    for (int r = 0; r < nq; r++) {
      Elem64Row &e = eb.rows[eb.count++];
      e = Elem64Row{};
      e.a1 = src[p] + static_cast<size_t>(r) * n;
      e.o0 = dst[p] + static_cast<size_t>(r) * n;
      e.q = P->primes[g[r]];
      if (eb.count == kMaxElem64Rows) {
        launch_permute64(eb, galois, stream);
        eb.count = 0;
      }
    }
  launch_permute64(eb, galois, stream);
  res.scale = a.scale;
  res.num_slots = a.num_slots;
  return check("permute64");
}

Status Context64::hrot_add(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key, int rot) {
  // HRotAdd (Context.cpp:800-830): HRot(a) + b
  CHD_CHECK(a.np == b.np, kErrShape, "HRotAdd: level mismatch");
  Ct64 t;
  CHD_TRY(hrot(t, a, key, rot));
  return add(res, t, b);
}

Status Context64::hconj_add(Ct64 &res, const Ct64 &a, const Ct64 &b, const Evk64 &key) {
  // HConjAdd (Context.cpp:832-860): HConj(a) + b
  CHD_CHECK(a.np == b.np, kErrShape, "HConjAdd: level mismatch");
  Ct64 t;
  CHD_TRY(hconj(t, a, key));
  return add(res, t, b);
}

Status Context64::mult_imag_unit(Ct64 &res, const Ct64 &a) {
  // ElementWise.cu:625-658: multiply by X^(N/2) = +-psi^(N/2)
  CHD_CHECK(a.np.aux == 0, kErrShape, "MultImaginaryUnit: no aux primes");
  const NP np = a.np;
  std::vector<int> g(np.total());
  P->gidx(np, g.data());
  std::vector<u64> k(np.total());
  for (int r = 0; r < np.total(); r++) k[r] = imag_unit[g[r]];
  const bool rx = a.has_rx;
  const u64 *pa[3] = {a.bx, a.ax, a.rx};
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, P->n, rx));
  u64 *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kMultImagUnit, np, rx ? 3 : 2, pd, pa, nullptr, k.data()));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context64::mult_const(Ct64 &res, const Ct64 &a, const u64 *cx, double cscale) {
  const NP np = a.np;
  const bool rx = a.has_rx;
  const u64 *pa[3] = {a.bx, a.ax, a.rx};
  const double sc = a.scale * cscale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, P->n, rx));
  u64 *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kMultConst, np, rx ? 3 : 2, pd, pa, nullptr, cx));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context64::add_const(Ct64 &res, const Ct64 &a, const u64 *cx) {
  // Context.cpp:174-203: the constant is added to bx, ax and rx are copied
  const NP np = a.np;
  const bool rx = a.has_rx;
  if (&res == &a && rx && !res.has_rx) return via_temp(res, [&](Ct64 &t) { return add_const(t, a, cx); });
  const u64 *keep[2] = {a.ax, a.rx};
  const u64 *pa[1] = {a.bx};
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, P->n, rx));
  u64 *pd[1] = {res.bx};
  CHD_TRY(elem_parts64(*this, Elem64Op::kAddConst, np, 1, pd, pa, nullptr, cx));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 8;
  if (keep[0] != res.ax) cudaMemcpyAsync(res.ax, keep[0], bytes, cudaMemcpyDeviceToDevice, stream);
  if (rx && keep[1] != res.rx) cudaMemcpyAsync(res.rx, keep[1], bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return check("add_const64");
}

Status Context64::level_down(Ct64 &res, const Ct64 &a, int target_level) {
  // LevelDown (Context.cpp:917-928): per level, times the constant 1 at
  // that level's scale, then Rescale
  CHD_CHECK(a.np.aux == 0 && !a.has_rx, kErrShape, "LevelDown: relinearised input without aux primes required");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0 && target_level >= 0 && level >= target_level, kErrInvalidLevel,
            "Invalid target level for LevelDown");
  CHD_CHECK(level <= P->spec.default_encryption_level, kErrInvalidLevel,
            "LevelDown: input above the default encryption level (no level-down constant there)");
  if (level == target_level) return copy(res, a);
  Ct64 cur, tmp;
  const Ct64 *prev = &a;
  std::vector<u64> cx;
  for (int i = level; i > target_level; i--) {
    encode_const(i, P->scale.at(i), 1.0, 0, &cx);
    CHD_TRY(mult_const(tmp, *prev, cx.data(), P->scale.at(i)));
    CHD_TRY(rescale(cur, tmp));
    prev = &cur;
  }
  res.swap(cur);
  return kOk;
}

}  // namespace w64
}  // namespace chd

// ------------------------------------------------------------------ C ABI
using namespace chd;
using namespace chd::w64;

struct chd64_context {
  std::unique_ptr<Context64> c;
};
struct chd64_ciphertext {
  Ct64 ct;
};
struct chd64_evk {
  Evk64 k;
};

namespace {
int fail64(int code, const std::string &m) {
  set_error(m);
  return code;
}
Status missing64(const char *what) {
  set_error(std::string(what) + ": null argument");
  return kErrInvalidArg;
}
}  // namespace

#define CHD64_CTX(ctx)                                                   \
  if (!(ctx)) return fail64(CHD_ERR_INVALID_ARG, "null context");        \
  DeviceGuard device_guard((ctx)->c->device)

extern "C" {

int chd64_context_create_json(const char *json, int device, chd64_context **out) try {
  if (!json || !out) return fail64(CHD_ERR_INVALID_ARG, "chd64_context_create_json: null argument");
  ParamSpec64 spec;
  std::string err;
  if (!parse_param_json64(json, &spec, &err)) return fail64(CHD_ERR_PARSE, err);
  int prev = 0;
  cudaGetDevice(&prev);
  auto c = std::make_unique<Context64>();
  const Status s = c->init(spec, device, &err);
  cudaSetDevice(prev);
  if (s != kOk) return fail64(s == kErrInvalidArg ? CHD_ERR_INVALID_ARG : CHD_ERR_CUDA, err);
  *out = new chd64_context{std::move(c)};
  return CHD_OK;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, std::string("chd64_context_create_json: ") + e.what());
}

void chd64_context_destroy(chd64_context *ctx) {
  if (!ctx) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->c->device);
  cudaStreamSynchronize(ctx->c->stream);
  delete ctx;
  cudaSetDevice(prev);
}

int chd64_context_synchronize(chd64_context *ctx) try {
  CHD64_CTX(ctx);
  const cudaError_t e = cudaStreamSynchronize(ctx->c->stream);
  return e == cudaSuccess ? CHD_OK : fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_context_set_stream(chd64_context *ctx, void *cuda_stream) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  cudaStreamSynchronize(C.stream);
  if (cuda_stream) {
    if (C.own_stream) cudaStreamDestroy(C.stream);
    C.own_stream = false;
    C.stream = static_cast<cudaStream_t>(cuda_stream);
  } else if (!C.own_stream) {
    cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking);
    C.own_stream = true;
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_max_level(const chd64_context *ctx) { return ctx ? ctx->c->P->max_level : -1; }
int chd64_alpha(const chd64_context *ctx) { return ctx ? ctx->c->P->alpha : -1; }

int chd64_level_np(const chd64_context *ctx, int level, int *num_main, int *num_ter) try {
  if (!ctx || !num_main || !num_ter) return fail64(CHD_ERR_INVALID_ARG, "chd64_level_np: null argument");
  if (level < 0 || level > ctx->c->P->max_level) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_level_np: invalid level");
  const NP np = ctx->c->P->level_np(level);
  *num_main = np.main;
  *num_ter = np.ter;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_primes(const chd64_context *ctx, uint64_t *out, int cap) {
  if (!ctx) return -1;
  const auto &p = ctx->c->P->primes;
  for (int i = 0; i < cap && i < static_cast<int>(p.size()); i++) out[i] = p[i];
  return static_cast<int>(p.size());
}

int chd64_ntt(chd64_context *ctx, int num_main, int num_ter, int num_aux, uint64_t *data_dev, int count, int inverse,
              int mont) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!data_dev || count < 1 || num_main < 0 || num_ter < 0 || num_aux < 0 || num_main > C.P->max_main ||
      num_ter > C.P->max_ter || num_aux > C.P->alpha)
    return fail64(CHD_ERR_INVALID_ARG, "chd64_ntt: invalid arguments");
  const NP np{num_main, num_ter, num_aux};
  const Status s = inverse ? C.intt(np, data_dev, count, mont != 0) : C.ntt(np, data_dev, count, mont != 0);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_modup_raw(chd64_context *ctx, int level, const uint64_t *src_dev, uint64_t *dst_dev) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!src_dev || !dst_dev) return fail64(CHD_ERR_INVALID_ARG, "chd64_modup_raw: null argument");
  if (level < 0 || level > C.P->max_level) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_modup_raw: invalid level");
  const Status s = C.modup(level, src_dev, dst_dev);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_moddown_raw(chd64_context *ctx, int level, int type, const uint64_t *src_dev, uint64_t *dst_dev,
                      int npoly) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!src_dev || !dst_dev || npoly < 1) return fail64(CHD_ERR_INVALID_ARG, "chd64_moddown_raw: invalid arguments");
  if (level < 0 || level > C.P->max_level) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_moddown_raw: invalid level");
  if (type < CHD_MODDOWN || type > CHD_MODDOWN_RESCALE)
    return fail64(CHD_ERR_INVALID_ARG, "chd64_moddown_raw: invalid type");
  const MDType t = type == CHD_MODDOWN ? MDType::kModDown : type == CHD_RESCALE ? MDType::kRescale
                                                                                   : MDType::kModDownRescale;
  const LevelMS64 &m = C.lms(level);
  const NP ns = C.P->level_np(level, t == MDType::kRescale ? 0 : m.num_aux);
  const NP nd = C.P->level_np(t == MDType::kModDown ? level : level - 1, 0);
  if (t != MDType::kModDown && level < 1) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_moddown_raw: no rescale at level 0");
  std::vector<const uint64_t *> s(npoly);
  std::vector<uint64_t *> d(npoly);
  for (int p = 0; p < npoly; p++) {
    s[p] = src_dev + static_cast<size_t>(p) * ns.total() * C.P->n;
    d[p] = dst_dev + static_cast<size_t>(p) * nd.total() * C.P->n;
  }
  const Status st = C.moddown(level, t, s.data(), d.data(), npoly);
  return st == kOk ? CHD_OK : st;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_create(chd64_context *ctx, chd64_ciphertext **out) {
  if (!ctx || !out) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_create: null argument");
  *out = new chd64_ciphertext();
  return CHD_OK;
}

void chd64_ct_destroy(chd64_ciphertext *ct) { delete ct; }

int chd64_ct_import(chd64_context *ctx, chd64_ciphertext *ct, int level, double scale, int num_slots,
                    const uint64_t *bx, const uint64_t *ax, int src_on_device) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!ct || !bx || !ax) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_import: null argument");
  if (level < 0 || level > C.P->max_level) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_ct_import: invalid level");
  const NP np = C.P->level_np(level);
  const Status s = ct->ct.reserve(np, C.P->n);
  if (s != kOk) return s;
  const size_t bytes = static_cast<size_t>(np.total()) * C.P->n * 8;
  const cudaMemcpyKind k = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(ct->ct.bx, bx, bytes, k, C.stream);
  cudaMemcpyAsync(ct->ct.ax, ax, bytes, k, C.stream);
  ct->ct.scale = scale;
  ct->ct.num_slots = num_slots;
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_export(chd64_context *ctx, const chd64_ciphertext *ct, uint64_t *bx, uint64_t *ax) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!ct || !bx || !ax) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_export: null argument");
  const size_t bytes = static_cast<size_t>(ct->ct.np.total()) * C.P->n * 8;
  cudaMemcpyAsync(bx, ct->ct.bx, bytes, cudaMemcpyDeviceToHost, C.stream);
  cudaMemcpyAsync(ax, ct->ct.ax, bytes, cudaMemcpyDeviceToHost, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_info(const chd64_ciphertext *ct, int *num_main, int *num_ter, double *scale, int *num_slots) {
  if (!ct) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_info: null argument");
  if (num_main) *num_main = ct->ct.np.main;
  if (num_ter) *num_ter = ct->ct.np.ter;
  if (scale) *scale = ct->ct.scale;
  if (num_slots) *num_slots = ct->ct.num_slots;
  return CHD_OK;
}

int chd64_evk_create(chd64_context *ctx, int beta, const uint64_t *bx, const uint64_t *ax, int src_on_device,
                     chd64_evk **out) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!bx || !ax || !out || beta < 1) return fail64(CHD_ERR_INVALID_ARG, "chd64_evk_create: invalid arguments");
  auto k = std::make_unique<chd64_evk>();
  k->k.np = NP{C.P->max_main, C.P->max_ter, C.P->alpha};
  k->k.beta = beta;
  const size_t bytes = static_cast<size_t>(beta) * k->k.np.total() * C.P->n * 8;
  if (cudaMalloc(&k->k.bx, bytes) != cudaSuccess || cudaMalloc(&k->k.ax, bytes) != cudaSuccess)
    return fail64(CHD_ERR_ALLOC, "chd64_evk_create: allocation failed");
  const cudaMemcpyKind kind = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(k->k.bx, bx, bytes, kind, C.stream);
  cudaMemcpyAsync(k->k.ax, ax, bytes, kind, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  if (e != cudaSuccess) return fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
  *out = k.release();
  return CHD_OK;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

void chd64_evk_destroy(chd64_evk *k) { delete k; }

int chd64_hmult(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
                const chd64_evk *key, int rescale) try {
  CHD64_CTX(ctx);
  if (!res || !a || !b || !key) return fail64(CHD_ERR_INVALID_ARG, "chd64_hmult: null argument");
  if (res == a || res == b) return fail64(CHD_ERR_INVALID_ARG, "chd64_hmult: the result must not alias an operand");
  const Status s = ctx->c->hmult(res->ct, a->ct, b->ct, key->k, rescale != 0);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_hrot(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key,
               int rot) try {
  CHD64_CTX(ctx);
  if (!res || !a || !key) return fail64(CHD_ERR_INVALID_ARG, "chd64_hrot: null argument");
  const Status s = ctx->c->hrot(res->ct, a->ct, key->k, rot);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_hconj(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key) try {
  CHD64_CTX(ctx);
  if (!res || !a || !key) return fail64(CHD_ERR_INVALID_ARG, "chd64_hconj: null argument");
  const Status s = ctx->c->hconj(res->ct, a->ct, key->k);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_rescale(chd64_context *ctx, chd64_ciphertext *res, const chd64_ciphertext *a) try {
  CHD64_CTX(ctx);
  if (!res || !a) return fail64(CHD_ERR_INVALID_ARG, "chd64_rescale: null argument");
  const Status s = ctx->c->rescale(res->ct, a->ct);
  return s == kOk ? CHD_OK : s;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_set_rx(chd64_context *ctx, chd64_ciphertext *ct, const uint64_t *rx, int src_on_device) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!ct || !rx) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_set_rx: null argument");
  if (!ct->ct.bx) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_set_rx: import bx and ax first");
  const NP np = ct->ct.np;
  // keep bx / ax: reserve grows only the rx buffer here
  const Status s = ct->ct.reserve(np, C.P->n, true);
  if (s != kOk) return s;
  const size_t bytes = static_cast<size_t>(np.total()) * C.P->n * 8;
  cudaMemcpyAsync(ct->ct.rx, rx, bytes, src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_export_rx(chd64_context *ctx, const chd64_ciphertext *ct, uint64_t *rx) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!ct || !rx) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_export_rx: null argument");
  if (!ct->ct.has_rx) return fail64(CHD_ERR_INVALID_ARG, "chd64_ct_export_rx: the ciphertext has no rx");
  const size_t bytes = static_cast<size_t>(ct->ct.np.total()) * C.P->n * 8;
  cudaMemcpyAsync(rx, ct->ct.rx, bytes, cudaMemcpyDeviceToHost, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : fail64(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

int chd64_ct_has_rx(const chd64_ciphertext *ct) { return ct ? (ct->ct.has_rx ? 1 : 0) : -1; }

double chd64_scale(const chd64_context *ctx, int level) {
  if (!ctx || level < 0 || level >= static_cast<int>(ctx->c->P->scale.size())) return 0.0;
  return ctx->c->P->scale[level];
}

int chd64_encode_const(chd64_context *ctx, int level, double scale, double value, int num_aux, uint64_t *cx) try {
  CHD64_CTX(ctx);
  Context64 &C = *ctx->c;
  if (!cx) return fail64(CHD_ERR_INVALID_ARG, "chd64_encode_const: null output");
  if (level < -1 || level > C.P->max_level) return fail64(CHD_ERR_INVALID_LEVEL, "chd64_encode_const: invalid level");
  if (num_aux < 0 || num_aux > C.P->alpha) return fail64(CHD_ERR_INVALID_ARG, "chd64_encode_const: invalid num_aux");
  std::vector<u64> v;
  C.encode_const(level, scale, value, num_aux, &v);
  std::memcpy(cx, v.data(), v.size() * 8);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail64(CHD_ERR_INTERNAL, e.what());
}

// Context<uint64_t> operations: null checks, then the operation's status
#define CHD64_OP(name, args, ...)                                         \
  int name args try {                                                     \
    CHD64_CTX(ctx);                                                       \
    if (!res || !a) return fail64(CHD_ERR_INVALID_ARG, #name ": null argument"); \
    const Status s = __VA_ARGS__;                                         \
    return s == kOk ? CHD_OK : s;                                         \
  } catch (const std::exception &e) {                                     \
    return fail64(CHD_ERR_INTERNAL, e.what());                            \
  }

CHD64_OP(chd64_copy, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a),
         ctx->c->copy(res->ct, a->ct))
CHD64_OP(chd64_neg, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a),
         ctx->c->neg(res->ct, a->ct))
CHD64_OP(chd64_mult_imaginary_unit, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a),
         ctx->c->mult_imag_unit(res->ct, a->ct))
CHD64_OP(chd64_add, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b),
         b ? ctx->c->add(res->ct, a->ct, b->ct) : missing64("chd64_add"))
CHD64_OP(chd64_sub, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b),
         b ? ctx->c->sub(res->ct, a->ct, b->ct) : missing64("chd64_sub"))
CHD64_OP(chd64_mult, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b),
         b ? ctx->c->mult_tensor(res->ct, a->ct, b->ct) : missing64("chd64_mult"))
CHD64_OP(chd64_relinearize,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key, int rescale),
         key ? ctx->c->relinearize(res->ct, a->ct, key->k, rescale != 0) : missing64("chd64_relinearize"))
CHD64_OP(chd64_mult_key, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_evk *key),
         key ? ctx->c->mult_key(res->ct, a->ct, key->k) : missing64("chd64_mult_key"))
CHD64_OP(chd64_permute,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, int rot, int conjugate),
         ctx->c->permute(res->ct, a->ct, rot, conjugate != 0))
CHD64_OP(chd64_hrot_add,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
          const chd64_evk *key, int rot),
         b && key ? ctx->c->hrot_add(res->ct, a->ct, b->ct, key->k, rot) : missing64("chd64_hrot_add"))
CHD64_OP(chd64_hconj_add,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const chd64_ciphertext *b,
          const chd64_evk *key),
         b && key ? ctx->c->hconj_add(res->ct, a->ct, b->ct, key->k) : missing64("chd64_hconj_add"))
CHD64_OP(chd64_mult_const,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const uint64_t *cx,
          double const_scale),
         cx ? ctx->c->mult_const(res->ct, a->ct, cx, const_scale) : missing64("chd64_mult_const"))
CHD64_OP(chd64_add_const, (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, const uint64_t *cx),
         cx ? ctx->c->add_const(res->ct, a->ct, cx) : missing64("chd64_add_const"))
CHD64_OP(chd64_level_down,
         (chd64_context * ctx, chd64_ciphertext *res, const chd64_ciphertext *a, int target_level),
         ctx->c->level_down(res->ct, a->ct, target_level))
#undef CHD64_OP

}  // extern "C"
