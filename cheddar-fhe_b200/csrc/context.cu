// Host orchestration of the CKKS evaluation core.
//
// The level model, ModSwitch constants and evaluator compositions follow the
// reference (scale-snu/cheddar-fhe): Parameter.cu:20-376, ModSwitch.cu:175-684,
// Context.cpp:62-949.  Everything that touches residues runs in the CUDA
// kernels of ntt.cu / elem.cu; this file only computes constants on the host
// and builds launch descriptors.
#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <limits>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>

#include "host.h"

namespace chd {

// ---------------------------------------------------------------- errors
namespace {
thread_local std::string g_error;
}
void set_error(const std::string &msg) { g_error = msg; }
const char *last_error() { return g_error.c_str(); }

// ---------------------------------------------------------- prime utilities
namespace prime {
uint32_t mul_mod(uint32_t a, uint32_t b, uint32_t q) {
  return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) % q);
}
uint32_t inv_mod(uint32_t a, uint32_t q) {
  int64_t t = 0, nt = 1, r = q, nr = a % q;
  while (nr) {
    int64_t k = r / nr;
    int64_t tmp = t - k * nt;
    t = nt;
    nt = tmp;
    tmp = r - k * nr;
    r = nr;
    nr = tmp;
  }
  if (t < 0) t += q;
  return static_cast<uint32_t>(t);
}
uint32_t pow_mod(uint32_t a, int64_t e, uint32_t q) {
  a %= q;
  if (e < 0) {
    a = inv_mod(a, q);
    e = -e;
  }
  uint64_t r = 1, b = a;
  while (e) {
    if (e & 1) r = (r * b) % q;
    b = (b * b) % q;
    e >>= 1;
  }
  return static_cast<uint32_t>(r);
}
uint32_t smallest_generator(uint32_t q) {
  // smallest r >= 2 whose order is q-1: r^((q-1)/f) != 1 for every prime
  // factor f of q-1 (the choice of generator fixes psi, which fixes the
  // evaluation order; it matches include/common/PrimeUtils.h:135-170)
  uint32_t phi = q - 1, t = phi;
  std::vector<uint32_t> f;
  for (uint32_t i = 2; static_cast<uint64_t>(i) * i <= t; i++) {
    if (t % i == 0) {
      f.push_back(i);
      while (t % i == 0) t /= i;
    }
  }
  if (t > 1) f.push_back(t);
  for (uint32_t r = 2; r < q; r++) {
    bool ok = true;
    for (uint32_t x : f)
      if (pow_mod(r, phi / x, q) == 1) {
        ok = false;
        break;
      }
    if (ok) return r;
  }
  return 0;
}
uint32_t primitive_root(uint32_t m, uint32_t q) { return pow_mod(smallest_generator(q), (q - 1) / m, q); }
int32_t inv_mod_word(uint32_t q) {
  uint32_t x = q;
  for (int i = 0; i < 5; i++) x *= 2u - q * x;
  return static_cast<int32_t>(x);
}
uint32_t to_mont(uint32_t a, uint32_t q) { return static_cast<uint32_t>((static_cast<uint64_t>(a) << 32) % q); }
int32_t centre(uint32_t a, uint32_t q) {
  return a > (q >> 1) ? static_cast<int32_t>(a) - static_cast<int32_t>(q) : static_cast<int32_t>(a);
}
}  // namespace prime

static unsigned brev_host(unsigned x, int bits) {
  unsigned r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// --------------------------------------------------------------- JSON
namespace {
struct JVal {
  enum T { kNull, kBool, kNum, kStr, kArr, kObj } t = kNull;
  double num = 0;
  bool b = false;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal *get(const std::string &k) const {
    for (auto &kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};
struct JParser {
  const std::string &s;
  size_t i = 0;
  std::string err;
  explicit JParser(const std::string &x) : s(x) {}
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\t' || s[i] == '\r')) i++;
  }
  bool val(JVal &v) {
    ws();
    if (i >= s.size()) return fail("unexpected end");
    char c = s[i];
    if (c == '{') {
      v.t = JVal::kObj;
      i++;
      ws();
      if (i < s.size() && s[i] == '}') {
        i++;
        return true;
      }
      while (true) {
        ws();
        JVal k;
        if (!str(k)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail("expected ':'");
        i++;
        JVal x;
        if (!val(x)) return false;
        v.obj.emplace_back(k.s, std::move(x));
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          i++;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.t = JVal::kArr;
      i++;
      ws();
      if (i < s.size() && s[i] == ']') {
        i++;
        return true;
      }
      while (true) {
        JVal x;
        if (!val(x)) return false;
        v.arr.push_back(std::move(x));
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          i++;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') return str(v);
    if (s.compare(i, 4, "true") == 0) {
      v.t = JVal::kBool;
      v.b = true;
      i += 4;
      return true;
    }
    if (s.compare(i, 5, "false") == 0) {
      v.t = JVal::kBool;
      i += 5;
      return true;
    }
    if (s.compare(i, 4, "null") == 0) {
      i += 4;
      return true;
    }
    size_t j = i;
    while (j < s.size() && (isdigit(static_cast<unsigned char>(s[j])) || s[j] == '-' || s[j] == '+' ||
                            s[j] == '.' || s[j] == 'e' || s[j] == 'E'))
      j++;
    if (j == i) return fail("unexpected character");
    v.t = JVal::kNum;
    v.s = s.substr(i, j - i);  // the token, for exact integers beyond a double
    v.num = std::strtod(v.s.c_str(), nullptr);
    i = j;
    return true;
  }
  bool str(JVal &v) {
    if (i >= s.size() || s[i] != '"') return fail("expected string");
    i++;
    v.t = JVal::kStr;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\' && i + 1 < s.size()) i++;
      v.s.push_back(s[i++]);
    }
    if (i >= s.size()) return fail("unterminated string");
    i++;
    return true;
  }
  bool fail(const char *m) {
    err = std::string(m) + " at offset " + std::to_string(i);
    return false;
  }
};
}  // namespace

template <typename W>
bool parse_spec(const std::string &text, ParamSpecT<W> *out, std::string *err) {
  // schema of unittest/Testbed.h:95-221 of the reference
  JParser p(text);
  JVal root;
  if (!p.val(root) || root.t != JVal::kObj) {
    *err = "JSON parse error: " + (p.err.empty() ? std::string("not an object") : p.err);
    return false;
  }
  auto num = [&](const char *k, double *v, bool req) -> bool {
    const JVal *x = root.get(k);
    if (!x) {
      if (req) *err = std::string("Missing ") + k + " in JSON";
      return !req;
    }
    if (x->t != JVal::kNum) {
      *err = std::string(k) + " should be a number";
      return false;
    }
    *v = x->num;
    return true;
  };
  auto primes = [&](const char *k, std::vector<W> *v, bool req) -> bool {
    const JVal *x = root.get(k);
    if (!x) {
      if (req) *err = std::string("Missing ") + k + " in JSON";
      return !req;
    }
    if (x->t != JVal::kArr) {
      *err = std::string(k) + " should be an array";
      return false;
    }
    for (auto &e : x->arr) {
      if (e.t != JVal::kNum || e.s.empty() || e.s.find_first_not_of("0123456789") != std::string::npos) {
        *err = std::string(k) + " should be an array of integers";
        return false;
      }
      errno = 0;
      const unsigned long long x = std::strtoull(e.s.c_str(), nullptr, 10);
      const bool big = errno == ERANGE || x > static_cast<unsigned long long>(std::numeric_limits<W>::max());
      v->push_back(big ? std::numeric_limits<W>::max() : static_cast<W>(x));
    }
    return true;
  };
  double d;
  ParamSpecT<W> s;
  if (!num("log_degree", &d, true)) return false;
  s.log_degree = static_cast<int>(d);
  if (!num("log_default_scale", &d, true)) return false;
  s.base_scale = std::ldexp(1.0, static_cast<int>(d));
  if (!num("default_encryption_level", &d, true)) return false;
  s.default_encryption_level = static_cast<int>(d);
  if (!primes("main_primes", &s.main_primes, true)) return false;
  if (!primes("terminal_primes", &s.ter_primes, false)) return false;
  if (!primes("auxiliary_primes", &s.aux_primes, true)) return false;
  const JVal *lc = root.get("level_config");
  if (!lc || lc->t != JVal::kArr) {
    *err = "Missing level_config in JSON";
    return false;
  }
  for (auto &e : lc->arr) {
    if (e.t != JVal::kArr || e.arr.size() != 2) {
      *err = "level_config should be an array of pairs";
      return false;
    }
    s.level_config.emplace_back(static_cast<int>(e.arr[0].num), static_cast<int>(e.arr[1].num));
  }
  if (const JVal *ab = root.get("additional_base")) {
    if (ab->t != JVal::kArr || ab->arr.size() != 2) {
      *err = "additional_base should be an array of pairs";
      return false;
    }
    s.additional_base = {static_cast<int>(ab->arr[0].num), static_cast<int>(ab->arr[1].num)};
  }
  if (num("dense_hamming_weight", &d, false) && root.get("dense_hamming_weight")) s.dense_hw = static_cast<int>(d);
  if (num("sparse_hamming_weight", &d, false) && root.get("sparse_hamming_weight")) s.sparse_hw = static_cast<int>(d);
  if (const JVal *b = root.get("boot")) s.boot = b->t == JVal::kBool && b->b;
  if (num("num_cts_levels", &d, false) && root.get("num_cts_levels")) s.num_cts_levels = static_cast<int>(d);
  if (num("num_stc_levels", &d, false) && root.get("num_stc_levels")) s.num_stc_levels = static_cast<int>(d);
  *out = s;
  return true;
}

bool parse_param_json(const std::string &text, ParamSpec *out, std::string *err) {
  return parse_spec(text, out, err);
}
bool parse_param_json64(const std::string &text, ParamSpec64 *out, std::string *err) {
  return parse_spec(text, out, err);
}

// -------------------------------------------------------------- Params
static bool np_less(std::pair<int, int> a, std::pair<int, int> b) {
  // Parameter.cu:10-15
  int at = a.first + a.second, bt = b.first + b.second;
  return at < bt || (at == bt && a.first < b.first);
}

std::unique_ptr<Params> Params::create(const ParamSpec &spec, std::string *err) {
  // validation of Parameter.cu:36-84
  if (spec.log_degree < 12 || spec.log_degree > 16) {
    *err = "log_degree must be in [12, 16]";
    return nullptr;
  }
  if (spec.main_primes.empty() || spec.aux_primes.empty() || spec.level_config.empty()) {
    *err = "main_primes, auxiliary_primes and level_config must be non-empty";
    return nullptr;
  }
  const uint32_t two_n = 2u << spec.log_degree;
  for (auto *lst : {&spec.main_primes, &spec.aux_primes, &spec.ter_primes})
    for (uint32_t p : *lst) {
      if (p >= (1u << 31)) {
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
    // the key switch and the per-limb descriptors of the kernels hold the
    // extended basis Q u P in 64-entry tables
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
  if (spec.default_encryption_level < 0 ||
      spec.default_encryption_level >= static_cast<int>(spec.level_config.size())) {
    *err = "Invalid default encryption level";
    return nullptr;
  }
  auto P = std::make_unique<Params>();
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
  P->short_np.aux = P->short_np.main + P->short_np.ter;
  if (P->short_np.main < 0 || P->short_np.ter < 0 || P->short_np.aux > na) {
    *err = "Invalid additional base configuration";
    return nullptr;
  }
  for (int i = nt - 1; i >= 0; i--) P->primes.push_back(spec.ter_primes[i]);
  for (uint32_t p : spec.main_primes) P->primes.push_back(p);
  for (uint32_t p : spec.aux_primes) P->primes.push_back(p);
  for (uint32_t p : P->primes) P->qinv.push_back(prime::inv_mod_word(p));
  P->galois.assign(P->n / 2 + 1, 1);
  for (int i = 1; i < P->n / 2; i++) P->galois[i] = static_cast<int>((static_cast<int64_t>(P->galois[i - 1]) * 5) % (2 * P->n));
  // scales, Parameter.cu:145-190
  P->rescale_prod.assign(P->max_level + 1, 0.0);
  P->scale.assign(spec.default_encryption_level + 1, 0.0);
  P->scale[0] = spec.base_scale;
  double ns = spec.base_scale;
  for (int i = 1; i <= P->max_level; i++) {
    NP up = P->level_np(i), lo = P->level_np(i - 1);
    int td = up.ter - lo.ter, md = up.main - lo.main;
    double num = 1.0, den = 1.0;
    if (td >= 0)
      for (int j = 0; j < td; j++) num *= spec.ter_primes[lo.ter + j];
    else
      for (int j = 0; j < -td; j++) den *= spec.ter_primes[up.ter + j];
    if (md >= 0)
      for (int j = 0; j < md; j++) num *= spec.main_primes[lo.main + j];
    else
      for (int j = 0; j < -md; j++) den *= spec.main_primes[up.main + j];
    P->rescale_prod[i] = num / den;
    if (i <= spec.default_encryption_level) {
      ns = std::sqrt(ns * P->rescale_prod[i]);
      P->scale[i] = ns;
    }
  }
  return P;
}

NP Params::level_np(int level, int num_aux) const {
  if (level == -1) return NP{short_np.main, short_np.ter, num_aux};
  auto c = spec.level_config.at(level);
  return NP{c.first, c.second, num_aux};
}

int Params::np_to_level(const NP &np) const {
  for (int l = 0; l <= max_level; l++)
    if (spec.level_config[l].first == np.main && spec.level_config[l].second == np.ter) return l;
  if (np.main == short_np.main && np.ter == short_np.ter) return -1;
  return -2;
}

void Params::gidx(const NP &np, int *out) const {
  int k = 0;
  for (int i = 0; i < np.q(); i++) out[k++] = max_ter - np.ter + i;
  for (int a = 0; a < np.aux; a++) out[k++] = L + a;
}

int Params::sse_num_aux() const {
  return spec.level_config[0].first + spec.level_config[0].second - spec.additional_base.first -
         spec.additional_base.second;
}

uint32_t Params::galois_of(int amount) const {
  if (amount == -1) return 2u * n - 1;
  return static_cast<uint32_t>(galois.at(amount));
}

// -------------------------------------------------------------- devices
DeviceCt::~DeviceCt() {
  if (owned) {
    cudaFree(bx);
    cudaFree(ax);
    cudaFree(rx);
  }
}

DeviceCt &DeviceCt::operator=(DeviceCt &&o) noexcept {
  if (this != &o) {
    if (owned) {
      cudaFree(bx);
      cudaFree(ax);
      cudaFree(rx);
    }
    take(o);
  }
  return *this;
}

Status DeviceCt::reserve(const NP &want, bool want_rx, int n) {
  size_t words = static_cast<size_t>(want.total()) * n;
  if (!owned) {
    CHD_CHECK(words <= cap_words && (!want_rx || rx), kErrShape, "wrapped ciphertext buffer too small");
  } else if (words > cap_words || (want_rx && !rx)) {
    size_t cap = std::max(words, cap_words);
    uint32_t *nb = nullptr, *na = nullptr, *nr = nullptr;
    if (cudaMalloc(&nb, cap * 4) != cudaSuccess || cudaMalloc(&na, cap * 4) != cudaSuccess ||
        (want_rx && cudaMalloc(&nr, cap * 4) != cudaSuccess)) {
      cudaFree(nb);
      cudaFree(na);
      set_error("device allocation failed");
      return kErrAlloc;
    }
    // reserve is only called before the result is written; old contents are
    // not needed.  The buffers are freed after the stream drains.
    cudaDeviceSynchronize();
    cudaFree(bx);
    cudaFree(ax);
    cudaFree(rx);
    bx = nb;
    ax = na;
    rx = nr;
    cap_words = cap;
  }
  np = want;
  has_rx = want_rx;
  return kOk;
}

DeviceEvk::~DeviceEvk() {
  if (owned) {
    cudaFree(bx);
    cudaFree(ax);
  }
}

Arena::~Arena() {
  for (auto &c : chunks_) cudaFree(c.p);
}

void *Arena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~static_cast<size_t>(255);
  // find the chunk holding top_
  for (auto &c : chunks_) {
    if (top_ >= c.start && top_ < c.start + c.size) {
      if (top_ + bytes <= c.start + c.size) {
        void *p = c.p + (top_ - c.start);
        top_ += bytes;
        return p;
      }
      break;
    }
  }
  // next chunk that fits entirely, starting after top_
  for (auto &c : chunks_) {
    if (c.start >= top_ && c.size >= bytes) {
      top_ = c.start + bytes;
      return c.p;
    }
  }
  size_t sz = std::max(bytes, total_ ? total_ : static_cast<size_t>(64) << 20);
  char *p = nullptr;
  if (cudaMalloc(&p, sz) != cudaSuccess) return nullptr;
  chunks_.push_back(Chunk{p, sz, total_});
  top_ = total_ + bytes;
  total_ += sz;
  return p;
}

void Arena::release(size_t m) { top_ = m; }


// -------------------------------------------------------------- Context
std::unique_ptr<Context> Context::create(const ParamSpec &spec, int device, std::string *err) {
  auto c = std::unique_ptr<Context>(new Context());
  if (c->init(spec, device, err) != kOk) return nullptr;
  return c;
}

Context::~Context() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto &m : ms) {
    for (auto *p : m.d_mod_up2) cudaFree(p);
    cudaFree(m.d_mod_down2);
    cudaFree(m.d_rs2);
    cudaFree(m.d_mdr2);
  }
  cudaFree(d_primes);
  cudaFree(d_qinv);
  cudaFree(d_err);
  cudaFree(d_tw);
  cudaFree(d_itw);
  cudaFree(d_enc_tw);
  cudaFree(d_galois);
  for (cudaEvent_t e : timer.ev) cudaEventDestroy(e);
  if (aux_stream) {
    cudaStreamSynchronize(aux_stream);
    cudaStreamDestroy(aux_stream);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

int Context::timer_mark() {
  if (!timer.on) return -1;
  if (timer.used == static_cast<int>(timer.ev.size())) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    timer.ev.push_back(e);
  }
  cudaEventRecord(timer.ev[timer.used], stream);
  return timer.used++;
}

void Context::timer_span(int stage, int e0, int launches) {
  if (e0 < 0) return;
  const int e1 = timer_mark();
  if (e1 >= 0) timer.spans.push_back({stage, e0, e1, launches});
}

Status Context::timer_read(double *ms, int *launches) {
  for (int s = 0; s < kKsStages; s++) {
    ms[s] = 0;
    launches[s] = 0;
  }
  for (const auto &sp : timer.spans) {
    CHD_CHECK(cudaEventSynchronize(timer.ev[sp.e1]) == cudaSuccess, kErrCuda, "stage timer: event wait failed");
    float t = 0;
    CHD_CHECK(cudaEventElapsedTime(&t, timer.ev[sp.e0], timer.ev[sp.e1]) == cudaSuccess, kErrCuda,
              "stage timer: elapsed time failed");
    ms[sp.stage] += t;
    launches[sp.stage] += sp.launches;
  }
  return kOk;
}

void Context::mont_as_shoup(uint32_t c, int g, uint32_t *w, uint32_t *ws) const {
  const uint32_t q = P->primes[g];
  *w = prime::mul_mod(c, r_inv[g], q);
  *ws = static_cast<uint32_t>((static_cast<uint64_t>(*w) << 32) / q);
}

Status Context::check_cuda(const char *where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

namespace {
// ModSwitch constant tables, ModSwitch.cu:320-370
void ms_consts(uint32_t n, const std::vector<uint32_t> &src, const std::vector<uint32_t> &dst, int rs, int re,
               std::vector<uint32_t> *c1, std::vector<int32_t> *c2) {
  const size_t sl = src.size(), dl = dst.size();
  c1->assign(sl, 1);
  c2->assign(sl * dl, 0);
  for (size_t i = 0; i < sl; i++) {
    uint32_t m = src[i], v = 1;
    for (size_t j = 0; j < sl; j++)
      if (j != i) v = prime::mul_mod(v, src[j], m);
    v = prime::inv_mod(prime::mul_mod(v, n, m), m);
    for (int j = rs; j < re; j++) v = prime::mul_mod(v, dst[j], m);
    (*c1)[i] = v;  // plain form: INTT output is x*R, the Montgomery product drops R
  }
  for (size_t mi = 0; mi < dl; mi++) {
    uint32_t p = dst[mi];
    for (size_t i = 0; i < sl; i++) {
      uint32_t acc = 1;
      for (size_t j = 0; j < sl; j++)
        if (j != i) acc = prime::mul_mod(acc, src[j], p);
      acc = prime::to_mont(prime::to_mont(acc, p), p);
      (*c2)[mi * sl + i] = prime::centre(acc, p);
    }
  }
}
// ModDown epilogue constants, ModSwitch.cu:372-411
void epi_consts(const std::vector<uint32_t> &src, const std::vector<uint32_t> &dst, int rs, int re,
                std::vector<uint32_t> *inv, std::vector<uint32_t> *pad) {
  const size_t dl = dst.size();
  inv->assign(dl, 0);
  for (size_t i = 0; i < dl; i++) {
    uint32_t p = dst[i], v = 1;
    for (uint32_t s : src) v = prime::mul_mod(v, s, p);
    (*inv)[i] = prime::to_mont(prime::inv_mod(v, p), p);
  }
  if (!pad) return;
  const int rl = re - rs;
  pad->assign(dl - rl, 0);
  for (int i = 0; i < static_cast<int>(dl) - rl; i++) {
    int pi = i >= rs ? i + rl : i;
    uint32_t p = dst[pi], v = 1;
    for (int j = rs; j < re; j++) v = prime::mul_mod(v, dst[j], p);
    (*pad)[i] = prime::to_mont(v, p);
  }
}
int32_t *upload_i32(const std::vector<int32_t> &v) {
  int32_t *p = nullptr;
  if (v.empty()) return nullptr;
  if (cudaMalloc(&p, v.size() * 4) != cudaSuccess) return nullptr;
  cudaMemcpy(p, v.data(), v.size() * 4, cudaMemcpyHostToDevice);
  return p;
}
}  // namespace

void build_level_ms(const Params &P, int level, LevelMS *out) {
  // ModSwitch.cu:175-318 of the reference
  LevelMS &m = *out;
  const uint32_t n = static_cast<uint32_t>(P.n);
  m.level = level;
  m.num_aux = level == -1 ? P.sse_num_aux() : P.alpha;
  NP np = P.level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  m.num_q = nq;
  m.beta = level == -1 ? 1 : (np.main + P.max_ter + m.num_aux - 1) / m.num_aux;
  std::vector<int> g(tot);
  P.gidx(np, g.data());
  std::vector<uint32_t> lp(tot);
  for (int i = 0; i < tot; i++) lp[i] = P.primes[g[i]];
  const int padded = level == -1 ? nq : np.main + P.max_ter;
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
    std::vector<uint32_t> src(lp.begin() + s, lp.begin() + e), dst(lp.begin(), lp.begin() + s);
    dst.insert(dst.end(), lp.begin() + e, lp.end());
    std::vector<uint32_t> c1;
    ms_consts(n, src, dst, 0, 0, &c1, &m.mod_up2[i]);
    std::copy(c1.begin(), c1.end(), m.mod_up1.begin() + s);
  }
  std::vector<uint32_t> qp(lp.begin(), lp.begin() + nq), pp(lp.begin() + nq, lp.end());
  ms_consts(n, pp, qp, 0, 0, &m.mod_down1, &m.mod_down2);
  epi_consts(pp, qp, 0, 0, &m.inv_p_prod, nullptr);
  if (level <= 0) return;
  NP nn = P.level_np(level - 1, m.num_aux);
  std::vector<int> gn(nn.total());
  P.gidx(nn, gn.data());
  std::vector<uint32_t> next(nn.q());
  for (int i = 0; i < nn.q(); i++) next[i] = P.primes[gn[i]];
  const int nnq = nn.q();
  const int md = np.main - nn.main, td = np.ter - nn.ter;
  std::vector<uint32_t> rs_src;
  if (td > 0) {
    if (md > 0) return;
    rs_src.assign(lp.begin(), lp.begin() + td);
    m.pad_start = 0;
    m.pad_end = nq - td;
    m.restore_start = nnq + md;
    m.restore_end = nnq;
  } else if (md > 0) {
    rs_src.assign(lp.begin() + nq - md, lp.begin() + nq);
    m.pad_start = -td;
    m.pad_end = nq - md - td;
    m.restore_start = 0;
    m.restore_end = -td;
  } else {
    return;
  }
  m.has_rescale = true;
  std::vector<uint32_t> mdr_src = rs_src;
  mdr_src.insert(mdr_src.end(), pp.begin(), pp.end());
  m.rs_src_len = static_cast<int>(rs_src.size());
  m.mdr_src_len = static_cast<int>(mdr_src.size());
  m.rs_dst_len = nnq;
  ms_consts(n, rs_src, next, m.restore_start, m.restore_end, &m.rs1, &m.rs2);
  epi_consts(rs_src, next, m.restore_start, m.restore_end, &m.rs_inv, &m.rs_pad);
  ms_consts(n, mdr_src, next, m.restore_start, m.restore_end, &m.mdr1, &m.mdr2);
  epi_consts(mdr_src, next, m.restore_start, m.restore_end, &m.mdr_inv, &m.mdr_pad);
}

Status Context::init(const ParamSpec &spec, int dev, std::string *err) {
  P = Params::create(spec, err);
  if (!P) return kErrInvalidArg;
  device = dev;
  if (cudaSetDevice(dev) != cudaSuccess) {
    *err = "cudaSetDevice failed";
    return kErrCuda;
  }
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    *err = "stream creation failed";
    return kErrCuda;
  }
  own_stream = true;
  if (cudaStreamCreateWithFlags(&aux_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess) {
    *err = "auxiliary stream creation failed";
    return kErrCuda;
  }
  if (const char *e = std::getenv("CHD_SPLIT_STREAMS")) split_streams = std::atoi(e) != 0;
  const int n = P->n, np_all = P->L + P->alpha;
  // twiddles, NTT.cu:1233-1299: psi_rev[j] = psi^brev(j); stored plain with
  // the Shoup companion floor(w 2^32 / q)
  std::vector<uint2> tw(static_cast<size_t>(np_all) * n), itw(tw.size());
  n_inv.resize(np_all);
  n_inv_mont.resize(np_all);
  mont_conv.resize(np_all);
  imag_unit.resize(np_all);
  r_inv.resize(np_all);
  std::vector<uint32_t> pw(n), pwi(n);
  auto shoup = [](uint32_t w, uint32_t q) { return static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / q); };
  for (int g = 0; g < np_all; g++) {
    uint32_t q = P->primes[g];
    uint32_t psi = prime::primitive_root(2u * n, q), psi_inv = prime::inv_mod(psi, q);
    n_inv[g] = prime::inv_mod(static_cast<uint32_t>(n), q);
    n_inv_mont[g] = prime::to_mont(n_inv[g], q);
    mont_conv[g] = prime::to_mont(prime::to_mont(1, q), q);
    r_inv[g] = prime::inv_mod(prime::to_mont(1, q), q);
    pw[0] = pwi[0] = 1;
    for (int j = 1; j < n; j++) {
      pw[j] = prime::mul_mod(pw[j - 1], psi, q);
      pwi[j] = prime::mul_mod(pwi[j - 1], psi_inv, q);
    }
    for (int j = 0; j < n; j++) {
      unsigned r = brev_host(j, P->log_n);
      tw[static_cast<size_t>(g) * n + j] = make_uint2(pw[r], shoup(pw[r], q));
      itw[static_cast<size_t>(g) * n + j] = make_uint2(pwi[r], shoup(pwi[r], q));
    }
    imag_unit[g] = prime::to_mont(pw[brev_host(1, P->log_n)], q);  // psi^(N/2), Montgomery
  }
  if (cudaMalloc(&d_primes, np_all * 4) != cudaSuccess || cudaMalloc(&d_qinv, np_all * 4) != cudaSuccess ||
      cudaMalloc(&d_tw, tw.size() * sizeof(uint2)) != cudaSuccess ||
      cudaMalloc(&d_itw, itw.size() * sizeof(uint2)) != cudaSuccess) {
    *err = "device allocation failed";
    return kErrAlloc;
  }
  if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess || cudaMemset(d_err, 0, sizeof(int)) != cudaSuccess) {
    *err = "device allocation failed";
    return kErrAlloc;
  }
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  cudaMemcpy(d_primes, P->primes.data(), np_all * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d_qinv, P->qinv.data(), np_all * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(uint2), cudaMemcpyHostToDevice);
  cudaMemcpy(d_itw, itw.data(), itw.size() * sizeof(uint2), cudaMemcpyHostToDevice);
  // P mod q_i (Montgomery), Context.cpp:78-90
  p_prod.resize(P->L);
  for (int i = 0; i < P->L; i++) {
    uint32_t q = P->primes[i], v = 1;
    for (int a = 0; a < P->alpha; a++) v = prime::mul_mod(v, P->primes[P->L + a], q);
    p_prod[i] = prime::to_mont(v, q);
  }
  // per-level ModSwitch constants, ModSwitch.cu:175-318
  ms.resize(P->max_level + 2);
  for (int level = -1; level <= P->max_level; level++) {
    LevelMS &m = ms[level + 1];
    build_level_ms(*P, level, &m);
    for (auto &t : m.mod_up2) m.d_mod_up2.push_back(t.empty() ? nullptr : upload_i32(t));
    m.d_mod_down2 = upload_i32(m.mod_down2);
    m.d_rs2 = upload_i32(m.rs2);
    m.d_mdr2 = upload_i32(m.mdr2);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    *err = std::string("context setup: ") + cudaGetErrorString(cudaGetLastError());
    return kErrCuda;
  }
  return kOk;
}

// ------------------------------------------------------- building blocks

Status Context::ntt(const NP &np, uint32_t *data, bool mont, int count, size_t stride) {
  const int tot = np.total(), n = P->n;
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  std::vector<RowDesc> rows;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < tot; i++) {
      RowDesc r{};
      r.src = r.dst = data + c * stride + static_cast<size_t>(i) * n;
      r.tw = tw(g[i]);
      r.q = P->primes[g[i]];
      mont_as_shoup(mont_conv[g[i]], g[i], &r.c0, &r.c0s);
      r.flags = mont ? kPreMult : 0u;
      rows.push_back(r);
    }
  return alternate_row_batches(rows, count > 1 && stride >= static_cast<size_t>(tot) * n,
                               [&](const RowBatch &rb, cudaStream_t s) { launch_ntt_fwd(rb, P->log_n, s); }, "ntt");
}

Status Context::alternate_row_batches(const std::vector<RowDesc> &rows, bool disjoint,
                                      const std::function<void(const RowBatch &, cudaStream_t)> &launch,
                                      const char *what) {
  // more rows than one launch takes: the launches alternate between the
  // context stream and aux_stream (forked and joined as in fork_halves), so
  // that one launch's column phase runs beside the other's row phase; rows
  // must be distinct limbs (disjoint), each transformed in place
  // launches of at most kAltRows rows alternate; fewer rows per launch
  // than kMaxRows interleave the two streams more finely (measured: 120)
  constexpr int kAltRows = 120;
  const bool split = split_streams && aux_stream != nullptr && disjoint &&
                     static_cast<int>(rows.size()) > kAltRows;
  if (!split) {
    for_row_batches(rows, [&](const RowBatch &rb) { launch(rb, stream); });
    return check_cuda(what);
  }
  CHD_CHECK(cudaEventRecord(ev_fork, stream) == cudaSuccess && cudaStreamWaitEvent(aux_stream, ev_fork, 0) == cudaSuccess,
            kErrCuda, "stream fork failed");
  int k = 0;
  for_row_batches(rows, [&](const RowBatch &rb) { launch(rb, (k++ & 1) ? aux_stream : stream); }, kAltRows);
  const bool joined =
      cudaEventRecord(ev_join, aux_stream) == cudaSuccess && cudaStreamWaitEvent(stream, ev_join, 0) == cudaSuccess;
  CHD_CHECK(joined, kErrCuda, "stream join failed");
  return check_cuda(what);
}

Status Context::intt(const NP &np, uint32_t *data, bool mont, int count, size_t stride) {
  const int tot = np.total(), n = P->n;
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  std::vector<RowDesc> rows;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < tot; i++) {
      RowDesc r{};
      r.src = r.dst = data + c * stride + static_cast<size_t>(i) * n;
      r.tw = itw(g[i]);
      r.q = P->primes[g[i]];
      mont_as_shoup(mont ? n_inv[g[i]] : n_inv_mont[g[i]], g[i], &r.c0, &r.c0s);
      rows.push_back(r);
    }
  return alternate_row_batches(rows, count > 1 && stride >= static_cast<size_t>(tot) * n,
                               [&](const RowBatch &rb, cudaStream_t s) { launch_ntt_inv(rb, P->log_n, s); }, "intt");
}

Status Context::bconv(const int32_t *xt, int K, const int32_t *table, const int *dst_gidx, int M, uint32_t *out) {
  CHD_CHECK(K >= 1 && K <= 16 && M >= 1 && M <= 64, kErrUnsupported, "bconv: K must be in [1,16], M in [1,64]");
  BConvBatch b{};
  b.count = 1;
  b.primes = d_primes;
  b.qinvs = d_qinv;
  BConvJob &j = b.jobs[0];
  j.xt = xt;
  j.out = out;
  j.table = table;
  j.K = K;
  j.M = M;
  for (int m = 0; m < M; m++) {
    j.out_row[m] = static_cast<uint8_t>(m);
    j.out_gidx[m] = static_cast<uint8_t>(dst_gidx[m]);
  }
  launch_bconv(b, P->log_n, stream);
  return check_cuda("bconv");
}

Status Context::bconv_many(int engine, int npoly, const int32_t *xt, int K, const std::vector<int32_t> &table,
                           const int *dst_gidx, int M, uint32_t *out) {
  CHD_CHECK(K >= 1 && K <= 16 && M >= 1 && M <= 64, kErrUnsupported, "bconv: K must be in [1,16], M in [1,64]");
  CHD_CHECK(static_cast<int>(table.size()) == M * K, kErrInvalidArg, "bconv: table size mismatch");
  if (npoly <= 0) return kOk;
  const size_t n = static_cast<size_t>(P->n);
  ArenaScope scope(arena);
  if (engine == 0) {
    int32_t *dt = static_cast<int32_t *>(arena.alloc(table.size() * 4));
    CHD_CHECK(dt, kErrAlloc, "bconv: scratch allocation failed");
    cudaMemcpyAsync(dt, table.data(), table.size() * 4, cudaMemcpyHostToDevice, stream);
    BConvBatch b{};
    b.primes = d_primes;
    b.qinvs = d_qinv;
    for (int i = 0; i < npoly; i++) {
      BConvJob &j = b.jobs[b.count++];
      j.xt = xt + static_cast<size_t>(i) * K * n;
      j.out = out + static_cast<size_t>(i) * M * n;
      j.table = dt;
      j.K = K;
      j.M = M;
      for (int m = 0; m < M; m++) {
        j.out_row[m] = static_cast<uint8_t>(m);
        j.out_gidx[m] = static_cast<uint8_t>(dst_gidx[m]);
      }
      if (b.count == kMaxBConvJobs) {
        launch_bconv(b, P->log_n, stream);
        b.count = 0;
      }
    }
    launch_bconv(b, P->log_n, stream);
    return check_cuda("bconv");
  }
  CHD_CHECK(engine == 1, kErrInvalidArg, "bconv: engine must be 0 (CUDA cores) or 1 (tensor cores)");
  CHD_CHECK(P->n % 128 == 0, kErrUnsupported, "bconv: tensor-core engine needs N >= 128");
  BConvTcDesc d{};
  d.K = K;
  d.M = M;
  d.n = P->n;
  d.npoly = npoly;
  d.ksteps = (4 * K + 31) / 32;
  d.nb = std::max(16, (4 * M + 15) / 16 * 16);
  // tiles per iteration: as many (up to 4) as keep the two accumulator
  // buffers within 128 TMEM columns, so that four CTAs share an SM (the
  // kernel is bound by the HBM loads in flight, not by the MMAs)
  d.tpi = 2 * 4 * d.nb <= 128 ? 4 : (2 * 2 * d.nb <= 128 ? 2 : 1);
  while ((P->n / 128) % d.tpi != 0) d.tpi /= 2;
  d.tmem_cols = 32;
  while (d.tmem_cols < 2 * d.tpi * d.nb) d.tmem_cols *= 2;
  // kind::i8: D s32 (bits 4-5 = 2), A s8 (bits 7-9 = 1), B u8 (bits 10-12 = 0),
  // both K-major, N >> 3 at bit 17, M >> 4 at bit 24
  d.idesc = (2u << 4) | (1u << 7) | (0u << 10) | (static_cast<uint32_t>(d.nb >> 3) << 17) | ((128u >> 4) << 24);
  // B operand image: row r = 4m + i (byte i of the constant), K byte kb = 4k + j
  std::vector<uint8_t> img(static_cast<size_t>(d.ksteps) * d.nb * 32, 0);
  for (int m = 0; m < M; m++) {
    const uint32_t p = P->primes[dst_gidx[m]];
    d.p[m] = p;
    d.pinv[m] = P->qinv[dst_gidx[m]];
    for (int k = 0; k < K; k++) {
      const int32_t tc = table[static_cast<size_t>(m) * K + k];
      const uint64_t t = tc < 0 ? static_cast<uint64_t>(static_cast<int64_t>(tc) + p) : static_cast<uint64_t>(tc);
      for (int j = 0; j < 4; j++) {
        const uint32_t c = static_cast<uint32_t>((t << (8 * j)) % p);
        const int kb = 4 * k + j;
        for (int i = 0; i < 4; i++) {
          const int r = 4 * m + i;
          const size_t off = static_cast<size_t>(kb / 32) * d.nb * 32 + (r / 8) * 256 + ((kb % 32) / 16) * 128 +
                             (r % 8) * 16 + (kb % 16);
          img[off] = static_cast<uint8_t>(c >> (8 * i));
        }
      }
    }
  }
  uint8_t *dimg = static_cast<uint8_t *>(arena.alloc(img.size()));
  CHD_CHECK(dimg, kErrAlloc, "bconv: scratch allocation failed");
  cudaMemcpyAsync(dimg, img.data(), img.size(), cudaMemcpyHostToDevice, stream);
  d.xt = xt;
  d.out = out;
  d.bmat = dimg;
  d.err = d_err;
  d.stall_polls = tc_stall_polls;
  const int rc = launch_bconv_tc(d, num_sms, stream);
  CHD_CHECK(rc == 0, kErrCuda, "bconv: tensor-core launch configuration failed");
  return check_cuda("bconv (tensor cores)");
}

Status Context::modup(int level, const uint32_t *src, uint32_t *const *dst) {
  const uint32_t *srcs[1] = {src};
  uint32_t *const *dsts[1] = {dst};
  return modup_many(level, 1, srcs, dsts);
}

Status Context::modup_many(int level, int count, const uint32_t *const *src, uint32_t *const *const *dst) {
  // ModSwitch.cu:429-509, for `count` independent inputs at one level
  const LevelMS &m = lms(level);
  const int n = P->n;
  NP np = P->level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  ArenaScope scope(arena);
  int32_t *xt = static_cast<int32_t *>(arena.alloc(static_cast<size_t>(count) * nq * n * 4));
  CHD_CHECK(xt, kErrAlloc, "modup: scratch allocation failed");
  if (P->log_n == 16) {
    uint32_t *rows_out = reinterpret_cast<uint32_t *>(xt);
    // two or more inputs: the halves on two streams (as the fused key
    // switch), each with its own part of the scratch, unless an output of
    // one half is an input of the other
    const int h = (count + 1) / 2;
    bool split = split_streams && aux_stream != nullptr && count >= 2;
    for (int c = 0; c < count && split; c++)
      for (int e = 0; e < count && split; e++)
        if ((c < h) != (e < h))
          for (int i = 0; i < m.beta; i++)
            if (m.dig_e[i] > 0 && dst[c][i] == src[e]) split = false;
    if (!split) return modup_fused(level, count, src, dst, rows_out);
    return fork_halves([&](bool second) {
      return second ? modup_fused(level, count - h, src + h, dst + h, rows_out + static_cast<size_t>(h) * nq * n)
                    : modup_fused(level, h, src, dst, rows_out);
    });
  }
  // 1. INTT * (N q-hat_i)^-1, centred (INTTAndMultConst with normalize)
  std::vector<RowDesc> rows;
  for (int c = 0; c < count; c++)
    for (int r = 0; r < nq; r++) {
      RowDesc d{};
      d.src = src[c] + static_cast<size_t>(r) * n;
      d.dst = reinterpret_cast<uint32_t *>(xt) + (static_cast<size_t>(c) * nq + r) * n;
      d.tw = itw(g[r]);
      d.q = P->primes[g[r]];
      mont_as_shoup(m.mod_up1[r], g[r], &d.c0, &d.c0s);
      d.flags = kCentre;
      rows.push_back(d);
    }
  for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_inv(rb, P->log_n, stream); });
  // 2. own primes copied, others base-converted
  BConvBatch b{};
  b.primes = d_primes;
  b.qinvs = d_qinv;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < m.beta; i++) {
      const int s = m.dig_s[i], e = m.dig_e[i];
      if (e <= 0) continue;
      cudaMemcpyAsync(dst[c][i] + static_cast<size_t>(s) * n, src[c] + static_cast<size_t>(s) * n,
                      static_cast<size_t>(e - s) * n * 4, cudaMemcpyDeviceToDevice, stream);
      BConvJob &j = b.jobs[b.count++];
      j.xt = xt + (static_cast<size_t>(c) * nq + s) * n;
      j.out = dst[c][i];
      j.table = m.d_mod_up2[i];
      j.K = e - s;
      j.M = tot - (e - s);
      CHD_CHECK(j.K <= 16 && j.M <= 64, kErrUnsupported, "modup: digit too large");
      int k = 0;
      for (int r = 0; r < tot; r++) {
        if (r >= s && r < e) continue;
        j.out_row[k] = static_cast<uint8_t>(r);
        j.out_gidx[k] = static_cast<uint8_t>(g[r]);
        k++;
      }
      if (b.count == kMaxBConvJobs) {
        launch_bconv(b, P->log_n, stream);
        b.count = 0;
      }
    }
  launch_bconv(b, P->log_n, stream);
  // 3. NTT of the converted rows (NTTForModUp)
  rows.clear();
  for (int c = 0; c < count; c++)
    for (int i = 0; i < m.beta; i++) {
      const int s = m.dig_s[i], e = m.dig_e[i];
      if (e <= 0) continue;
      for (int r = 0; r < tot; r++) {
        if (r >= s && r < e) continue;
        RowDesc d{};
        d.src = d.dst = dst[c][i] + static_cast<size_t>(r) * n;
        d.tw = tw(g[r]);
        d.q = P->primes[g[r]];
        rows.push_back(d);
      }
    }
  for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_fwd(rb, P->log_n, stream); });
  return check_cuda("modup");
}

// N = 2^16: INTT row phase -> fused column pass (INTT columns, centred
// constant, BConv, NTT columns) -> NTT row phase.
Status Context::modup_fused(int level, int count, const uint32_t *const *src, uint32_t *const *const *dst,
                            uint32_t *rows_out) {
  const LevelMS &m = lms(level);
  const int n = P->n;
  NP np = P->level_np(level, m.num_aux);
  const int nq = np.q(), tot = np.total();
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  std::vector<RowDesc> rows;
  for (int c = 0; c < count; c++)
    for (int r = 0; r < nq; r++) {
      RowDesc d{};
      d.src = src[c] + static_cast<size_t>(r) * n;
      d.dst = rows_out + (static_cast<size_t>(c) * nq + r) * n;
      d.tw = itw(g[r]);
      d.q = P->primes[g[r]];
      rows.push_back(d);
    }
  for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_inv_rows(rb, P->log_n, stream); });
  MSColBatch b{};
  b.engine = ks_engine;
  b.err = d_err;
  b.tw = d_tw;
  b.itw = d_itw;
  b.primes = d_primes;
  b.qinvs = d_qinv;
  for (int c = 0; c < count; c++)
    for (int i = 0; i < m.beta; i++) {
      const int s = m.dig_s[i], e = m.dig_e[i];
      if (e <= 0) continue;
      cudaMemcpyAsync(dst[c][i] + static_cast<size_t>(s) * n, src[c] + static_cast<size_t>(s) * n,
                      static_cast<size_t>(e - s) * n * 4, cudaMemcpyDeviceToDevice, stream);
      MSColJob &j = b.jobs[b.count++];
      j.src = rows_out + static_cast<size_t>(c) * nq * n;
      j.dst = dst[c][i];
      j.table = m.d_mod_up2[i];
      j.K = e - s;
      j.M = tot - (e - s);
      CHD_CHECK(j.K <= 16 && j.M <= 64, kErrUnsupported, "modup: digit too large");
      for (int k = 0; k < j.K; k++) {
        j.src_row[k] = static_cast<uint8_t>(s + k);
        j.src_gidx[k] = static_cast<uint8_t>(g[s + k]);
        mont_as_shoup(m.mod_up1[s + k], g[s + k], &j.c0[k], &j.c0s[k]);
      }
      int k = 0;
      for (int r = 0; r < tot; r++) {
        if (r >= s && r < e) continue;
        j.dst_row[k] = static_cast<uint8_t>(r);
        j.dst_gidx[k] = static_cast<uint8_t>(g[r]);
        k++;
      }
      if (b.count == kMaxMSColJobs) {
        launch_modswitch_cols(b, P->log_n, stream);
        b.count = 0;
      }
    }
  launch_modswitch_cols(b, P->log_n, stream);
  rows.clear();
  for (int c = 0; c < count; c++)
    for (int i = 0; i < m.beta; i++) {
      const int s = m.dig_s[i], e = m.dig_e[i];
      if (e <= 0) continue;
      for (int r = 0; r < tot; r++) {
        if (r >= s && r < e) continue;
        RowDesc d{};
        d.src = d.dst = dst[c][i] + static_cast<size_t>(r) * n;
        d.tw = tw(g[r]);
        d.q = P->primes[g[r]];
        rows.push_back(d);
      }
    }
  for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_fwd_rows(rb, P->log_n, stream); });
  return check_cuda("modup");
}

Status Context::moddown_plan(int level, MDType type, MDPlan *pl) const {
  const LevelMS &m = lms(level);
  CHD_CHECK(type == MDType::kModDown || m.has_rescale, kErrInvalidLevel, "rescale not available at this level");
  const int nsa = type == MDType::kRescale ? 0 : m.num_aux;
  pl->ns = P->level_np(level, nsa);
  pl->nd = P->level_np(type == MDType::kModDown ? level : level - 1, 0);
  pl->nn = NP{std::min(pl->ns.main, pl->nd.main), std::min(pl->ns.ter, pl->nd.ter), 0};
  pl->src_len = pl->ns.total() - pl->nn.total();
  pl->dst_len = pl->nd.total();
  CHD_CHECK(pl->src_len >= 1 && pl->src_len <= 16, kErrUnsupported, "moddown: more than 16 dropped primes");
  pl->c1 = type == MDType::kModDown ? m.mod_down1.data() : type == MDType::kRescale ? m.rs1.data() : m.mdr1.data();
  pl->table = type == MDType::kModDown ? m.d_mod_down2 : type == MDType::kRescale ? m.d_rs2 : m.d_mdr2;
  pl->inv = type == MDType::kModDown ? m.inv_p_prod.data() : type == MDType::kRescale ? m.rs_inv.data() : m.mdr_inv.data();
  pl->pad = type == MDType::kModDown ? nullptr : type == MDType::kRescale ? m.rs_pad.data() : m.mdr_pad.data();
  pl->gs.assign(pl->ns.total(), 0);
  pl->gd.assign(pl->nd.total(), 0);
  P->gidx(pl->ns, pl->gs.data());
  P->gidx(pl->nd, pl->gd.data());
  pl->srows.clear();
  const bool on_main = pl->ns.main > pl->nn.main, on_ter = pl->ns.ter > pl->nn.ter;
  CHD_CHECK(!(on_main && on_ter), kErrInvalidArg, "moddown: invalid prime combination");
  if (!on_ter)
    for (int r = pl->ns.ter + pl->nn.main; r < pl->ns.q(); r++) pl->srows.push_back(r);
  else
    for (int r = 0; r < pl->ns.ter - pl->nn.ter; r++) pl->srows.push_back(r);
  for (int a = 0; a < nsa; a++) pl->srows.push_back(pl->ns.q() + a);
  CHD_CHECK(static_cast<int>(pl->srows.size()) == pl->src_len, kErrInvalidArg, "moddown: internal row mismatch");
  pl->src2_start = pl->nd.ter - pl->nn.ter;
  pl->src2_end = pl->src2_start + pl->nn.q();
  pl->src2_off = std::max(0, pl->ns.ter - pl->nd.ter);
  return kOk;
}

Status Context::key_switch_fused(int level, int count, const KSIn *in, const DeviceEvk &key, MDType type,
                                 bool keep_ext) {
  std::vector<int> levels(std::max(count, 0), level);
  return key_switch_fused_levels(levels.data(), count, in, key, type, keep_ext);
}

Status Context::key_switch_fused_levels(const int *levels, int count, const KSIn *in, const DeviceEvk &key,
                                        MDType type, bool keep_ext) {
  // Two halves on two streams when the batch has at least two inputs and no
  // result of one half is an operand or a result of the other (with the
  // stage timer on, each half's spans are recorded on its own stream)
  bool split = split_streams && count >= 2 && aux_stream != nullptr;
  const int h = (count + 1) / 2;
  if (split) {
    auto ptrs_in = [&](int c, const void *p) {
      const KSIn &x = in[c];
      return p == x.b1 || p == x.a1 || p == x.b2 || p == x.a2 || p == x.out_b || p == x.out_a;
    };
    for (int c = 0; c < h && split; c++)
      for (int e = h; e < count && split; e++)
        if (ptrs_in(e, in[c].out_b) || ptrs_in(e, in[c].out_a) || ptrs_in(c, in[e].out_b) || ptrs_in(c, in[e].out_a))
          split = false;
  }
  if (!split) return key_switch_fused_pipeline(levels, count, in, key, type, keep_ext, false);
  return fork_halves([&](bool second) {
    return second ? key_switch_fused_pipeline(levels + h, count - h, in + h, key, type, keep_ext, true)
                  : key_switch_fused_pipeline(levels, h, in, key, type, keep_ext, true);
  });
}

Status Context::key_switch_fused_pipeline(const int *levels, int count, const KSIn *in, const DeviceEvk &key,
                                          MDType type, bool keep_ext, bool hold) {
  CHD_CHECK(P->log_n == 16, kErrUnsupported, "fused key switch needs N = 2^16");
  CHD_CHECK(keep_ext || type != MDType::kRescale, kErrInvalidArg,
            "fused key switch ends in ModDown or ModDownAndRescale");
  CHD_CHECK(key.np.aux == P->alpha && key.np.q() == P->L, kErrKey, "key switch: key basis mismatch");
  if (count <= 0) return kOk;
  // per-level shapes, shared by the ciphertexts at that level
  struct Shape {
    const LevelMS *m;
    int nq, tot, prime_offset;
    std::vector<int> g, digits;
    MDPlan pl;
  };
  std::map<int, Shape> shapes;
  for (int c = 0; c < count; c++) {
    const int level = levels[c];
    if (shapes.count(level)) continue;
    CHD_CHECK(level >= 0 && level <= P->max_level, kErrInvalidLevel, "key switch: invalid level");
    Shape &sh = shapes[level];
    sh.m = &lms(level);
    const NP np = P->level_np(level, P->alpha);
    sh.nq = np.q();
    sh.tot = np.total();
    CHD_CHECK(sh.tot <= 64 && sh.m->beta <= 8, kErrUnsupported, "key switch: more than 64 primes or 8 digits");
    sh.prime_offset = P->max_ter - np.ter;
    sh.g.resize(sh.tot);
    P->gidx(np, sh.g.data());
    for (int i = 0; i < sh.m->beta; i++)
      if (sh.m->dig_e[i] > 0) {
        CHD_CHECK(i < key.beta, kErrKey, "key switch: key has too few digits");
        sh.digits.push_back(i);
      }
    if (!keep_ext) CHD_TRY(moddown_plan(level, type, &sh.pl));
  }
  const int mode = in[0].mode;
  for (int c = 0; c < count; c++)
    CHD_CHECK(in[c].mode == mode, kErrInvalidArg, "key switch: mixed modes in one batch");
  // scratch offsets (in polynomials of N words) per ciphertext
  const size_t N = static_cast<size_t>(P->n);
  std::vector<size_t> o_t1(count), o_mu(count), o_acc(count), o_drop(count);
  size_t n_t1 = 0, n_mu = 0, n_acc = 0, n_drop = 0;
  for (int c = 0; c < count; c++) {
    const Shape &sh = shapes[levels[c]];
    o_t1[c] = n_t1;
    n_t1 += sh.nq;
    o_mu[c] = n_mu;
    n_mu += sh.digits.size() * sh.tot;
    o_acc[c] = n_acc;
    o_drop[c] = n_drop;
    if (!keep_ext) {
      n_acc += 2 * sh.tot;
      n_drop += 2 * sh.pl.src_len;
    }
  }
  HeldScope scope(arena, hold);
  uint32_t *t1 = static_cast<uint32_t *>(arena.alloc(n_t1 * N * 4));
  uint32_t *mu = static_cast<uint32_t *>(arena.alloc(n_mu * N * 4));
  // keep_ext: the accumulators go straight to the callers' buffers and
  // nothing is dropped
  uint32_t *acc = keep_ext ? nullptr : static_cast<uint32_t *>(arena.alloc(n_acc * N * 4));
  uint32_t *drop = keep_ext ? nullptr : static_cast<uint32_t *>(arena.alloc(n_drop * N * 4));
  CHD_CHECK(t1 && mu && (keep_ext || (acc && drop)), kErrAlloc, "key switch: scratch allocation failed");
  auto MU = [&](int c, int b) { return mu + (o_mu[c] + static_cast<size_t>(b) * shapes[levels[c]].tot) * N; };
  // 1. ModUp INTT row phase of the key-switched input (a1 a2 / ax / rx)
  std::vector<RowDesc> rows;
  for (int c = 0; c < count; c++) {
    const Shape &sh = shapes[levels[c]];
    for (int r = 0; r < sh.nq; r++) {
      RowDesc d{};
      const size_t o = static_cast<size_t>(r) * N;
      d.src = (in[c].mode == 2 ? in[c].a2 : in[c].a1) + o;
      if (in[c].mode == 0) {
        d.src2 = in[c].a2 + o;
        d.flags = kMulSrc2;
        d.qinv = P->qinv[sh.g[r]];
      }
      d.dst = t1 + (o_t1[c] + r) * N;
      d.tw = itw(sh.g[r]);
      d.q = P->primes[sh.g[r]];
      rows.push_back(d);
    }
  }
  int nl = 0, t0 = timer_mark();
  for_row_batches(rows, [&](const RowBatch &rb) {
    launch_ntt_inv_rows(rb, P->log_n, stream);
    nl++;
  });
  timer_span(kKsInvRows, t0, nl);
  MSColBatch b{};
  b.engine = ks_engine;
  b.err = d_err;
  b.tw = d_tw;
  b.itw = d_itw;
  b.primes = d_primes;
  b.qinvs = d_qinv;
  // 2. ModUp column pass per (ciphertext, digit)
  {
    nl = 0;
    t0 = timer_mark();
    b.count = 0;
    for (int c = 0; c < count; c++) {
      const Shape &sh = shapes[levels[c]];
      const LevelMS &m = *sh.m;
      for (size_t bi = 0; bi < sh.digits.size(); bi++) {
        const int i = sh.digits[bi], s = m.dig_s[i], e = m.dig_e[i];
        MSColJob &j = b.jobs[b.count++];
        j.src = t1 + o_t1[c] * N;
        j.dst = MU(c, static_cast<int>(bi));
        j.table = m.d_mod_up2[i];
        j.K = e - s;
        j.M = sh.tot - (e - s);
        CHD_CHECK(j.K <= 16 && j.M <= 64, kErrUnsupported, "modup: digit too large");
        for (int k = 0; k < j.K; k++) {
          j.src_row[k] = static_cast<uint8_t>(s + k);
          j.src_gidx[k] = static_cast<uint8_t>(sh.g[s + k]);
          mont_as_shoup(m.mod_up1[s + k], sh.g[s + k], &j.c0[k], &j.c0s[k]);
        }
        int k = 0;
        for (int r = 0; r < sh.tot; r++) {
          if (r >= s && r < e) continue;
          j.dst_row[k] = static_cast<uint8_t>(r);
          j.dst_gidx[k] = static_cast<uint8_t>(sh.g[r]);
          k++;
        }
        if (b.count == kMaxMSColJobs) {
          launch_modswitch_cols(b, P->log_n, stream);
          nl++;
          b.count = 0;
        }
      }
    }
    launch_modswitch_cols(b, P->log_n, stream);
    timer_span(kKsModUpCols, t0, nl + (b.count > 0));
  }
  // 3. row pass: ModUp NTT rows, key inner product, P (d0, d1), INTT rows of
  //    the dropped primes; a launch takes up to kMaxKSRowsCts ciphertexts
  //    over up to kMaxKSRowsLevels levels
  {
    const size_t kstride = static_cast<size_t>(key.np.total()) * N;
    auto fill_level = [&](int level, KSRowsLevel &lv) {
      const Shape &sh = shapes[level];
      const LevelMS &m = *sh.m;
      const int nb = static_cast<int>(sh.digits.size());
      for (int bi = 0; bi < nb; bi++) {
        lv.kb[bi] = key.bx + sh.digits[bi] * kstride;
        lv.ka[bi] = key.ax + sh.digits[bi] * kstride;
      }
      lv.beta = nb;
      lv.rows = sh.tot;
      lv.nq = sh.nq;
      for (int r = 0; r < sh.tot; r++) {
        lv.p_prod[r] = r < sh.nq ? p_prod[sh.prime_offset + r] : 0;
        lv.key_row[r] = static_cast<int16_t>(r < sh.nq ? sh.prime_offset + r : P->L + (r - sh.nq));
        lv.gidx[r] = static_cast<uint8_t>(sh.g[r]);
        lv.own_digit[r] = -1;
        lv.drop_idx[r] = -1;
        for (int bi = 0; bi < nb; bi++)
          if (r >= m.dig_s[sh.digits[bi]] && r < m.dig_e[sh.digits[bi]]) lv.own_digit[r] = static_cast<int8_t>(bi);
      }
      if (!keep_ext)
        for (int i = 0; i < sh.pl.src_len; i++) lv.drop_idx[sh.pl.srows[i]] = static_cast<int8_t>(i);
    };
    KSRowsDesc d{};
    d.tw = d_tw;
    d.itw = d_itw;
    d.primes = d_primes;
    d.qinvs = d_qinv;
    d.mode = mode;
    std::map<int, int> lv_of;  // level -> entry of d.lv in the launch being built
    nl = 0;
    t0 = timer_mark();
    auto flush = [&]() {
      if (d.count == 0) return;
      launch_ks_rows(d, P->log_n, stream, ks_engine == 2);
      nl++;
      d.count = d.nlv = d.max_rows = 0;
      lv_of.clear();
    };
    for (int c = 0; c < count; c++) {
      const int level = levels[c];
      if (d.count == kMaxKSRowsCts || (!lv_of.count(level) && d.nlv == kMaxKSRowsLevels)) flush();
      auto it = lv_of.find(level);
      if (it == lv_of.end()) {
        KSRowsLevel &lv = d.lv[d.nlv];
        lv = KSRowsLevel{};
        fill_level(level, lv);
        d.max_rows = std::max(d.max_rows, lv.rows);
        it = lv_of.emplace(level, d.nlv++).first;
      }
      const Shape &sh = shapes[level];
      const KSIn &x = in[c];
      KSRowsCt &k = d.ct[d.count++];
      k = KSRowsCt{};
      k.lv = it->second;
      for (size_t bi = 0; bi < sh.digits.size(); bi++) k.mu[bi] = MU(c, static_cast<int>(bi));
      k.b1 = x.b1;
      k.a1 = x.a1;
      k.b2 = x.b2;
      k.a2 = x.a2;
      if (keep_ext) {
        k.acc_b = x.out_b;
        k.acc_a = x.out_a;
      } else {
        k.acc_b = acc + o_acc[c] * N;
        k.acc_a = k.acc_b + static_cast<size_t>(sh.tot) * N;
        k.drop_b = drop + o_drop[c] * N;
        k.drop_a = k.drop_b + static_cast<size_t>(sh.pl.src_len) * N;
      }
    }
    flush();
    timer_span(kKsRows, t0, nl);
  }
  if (keep_ext) return check_cuda("key switch");
  // 4. ModDown column pass per (ciphertext, part)
  {
    nl = 0;
    t0 = timer_mark();
    b.count = 0;
    for (int c = 0; c < count; c++) {
      const MDPlan &pl = shapes[levels[c]].pl;
      for (int p = 0; p < 2; p++) {
        MSColJob &j = b.jobs[b.count++];
        j.src = drop + (o_drop[c] + static_cast<size_t>(p) * pl.src_len) * N;
        j.dst = p == 0 ? in[c].out_b : in[c].out_a;
        j.table = pl.table;
        j.K = pl.src_len;
        j.M = pl.dst_len;
        for (int i = 0; i < pl.src_len; i++) {
          const int gg = pl.gs[pl.srows[i]];
          j.src_row[i] = static_cast<uint8_t>(i);
          j.src_gidx[i] = static_cast<uint8_t>(gg);
          mont_as_shoup(pl.c1[i], gg, &j.c0[i], &j.c0s[i]);
        }
        for (int y = 0; y < pl.dst_len; y++) {
          j.dst_row[y] = static_cast<uint8_t>(y);
          j.dst_gidx[y] = static_cast<uint8_t>(pl.gd[y]);
        }
        if (b.count == kMaxMSColJobs) {
          launch_modswitch_cols(b, P->log_n, stream);
          nl++;
          b.count = 0;
        }
      }
    }
    launch_modswitch_cols(b, P->log_n, stream);
    timer_span(kKsModDownCols, t0, nl + (b.count > 0));
  }
  // 5. NTT row phase with the ModDown epilogue (src2 = kept accumulators)
  rows.clear();
  for (int c = 0; c < count; c++) {
    const Shape &sh = shapes[levels[c]];
    const MDPlan &pl = sh.pl;
    for (int p = 0; p < 2; p++) {
      const uint32_t *src = acc + (o_acc[c] + static_cast<size_t>(p) * sh.tot) * N;
      uint32_t *dst = p == 0 ? in[c].out_b : in[c].out_a;
      for (int y = 0; y < pl.dst_len; y++) {
        RowDesc d{};
        d.src = d.dst = dst + static_cast<size_t>(y) * N;
        d.tw = tw(pl.gd[y]);
        d.q = P->primes[pl.gd[y]];
        mont_as_shoup(pl.inv[y], pl.gd[y], &d.c2, &d.c2s);
        d.flags = kModDownEpi;
        if (y >= pl.src2_start && y < pl.src2_end) {
          d.flags |= kHasSrc2;
          d.src2 = src + static_cast<size_t>(pl.src2_off + y - pl.src2_start) * N;
          if (pl.pad) {
            d.flags |= kPadSrc2;
            mont_as_shoup(pl.pad[y - pl.src2_start], pl.gd[y], &d.c1, &d.c1s);
          }
        }
        rows.push_back(d);
      }
    }
  }
  nl = 0;
  t0 = timer_mark();
  for_row_batches(rows, [&](const RowBatch &rb) {
    launch_ntt_fwd_rows(rb, P->log_n, stream);
    nl++;
  });
  timer_span(kKsFwdRows, t0, nl);
  return check_cuda("key switch");
}

Status Context::moddown(int level, MDType type, const uint32_t *const *src, uint32_t *const *dst, int npoly) {
  // at N = 2^16 four or more polynomials run as two halves on two streams
  // (as the fused key switch does), unless a result of one half is an
  // operand or a result of the other
  bool split = split_streams && P->log_n == 16 && npoly >= 4 && aux_stream != nullptr;
  const int h = (npoly + 1) / 2;
  for (int p = 0; p < h && split; p++)
    for (int e = h; e < npoly && split; e++)
      if (dst[p] == src[e] || dst[p] == dst[e] || dst[e] == src[p]) split = false;
  if (!split) return moddown_pipeline(level, type, src, dst, npoly, false);
  return fork_halves([&](bool second) {
    return second ? moddown_pipeline(level, type, src + h, dst + h, npoly - h, true)
                  : moddown_pipeline(level, type, src, dst, h, true);
  });
}

Status Context::fork_halves(const std::function<Status(bool)> &half) {
  // the halves' scratch stays allocated until both are enqueued; later work
  // on the context stream is ordered after the join
  ArenaScope scope(arena);
  CHD_CHECK(cudaEventRecord(ev_fork, stream) == cudaSuccess && cudaStreamWaitEvent(aux_stream, ev_fork, 0) == cudaSuccess,
            kErrCuda, "stream fork failed");
  Status st = half(false);
  if (st == kOk) {
    cudaStream_t main_stream = stream;
    stream = aux_stream;
    st = half(true);
    stream = main_stream;
  }
  // the join is recorded on every path, so that nothing later on the
  // context stream overtakes work already enqueued on the auxiliary one
  const bool joined =
      cudaEventRecord(ev_join, aux_stream) == cudaSuccess && cudaStreamWaitEvent(stream, ev_join, 0) == cudaSuccess;
  CHD_TRY(st);
  CHD_CHECK(joined, kErrCuda, "stream join failed");
  return kOk;
}

Status Context::moddown_pipeline(int level, MDType type, const uint32_t *const *src, uint32_t *const *dst, int npoly,
                                 bool hold) {
  // ModSwitch.cu:566-684 with NTT.cu:973-1128 and the fused epilogue of
  // NTT.cu:456-601
  const LevelMS &m = lms(level);
  const int n = P->n;
  CHD_CHECK(type == MDType::kModDown || m.has_rescale, kErrInvalidLevel, "rescale not available at this level");
  const int nsa = type == MDType::kRescale ? 0 : m.num_aux;
  NP ns = P->level_np(level, nsa);
  NP nd = P->level_np(type == MDType::kModDown ? level : level - 1, 0);
  NP nn{std::min(ns.main, nd.main), std::min(ns.ter, nd.ter), 0};
  const int src_len = ns.total() - nn.total(), dst_len = nd.total();
  CHD_CHECK(src_len >= 1 && src_len <= 16, kErrUnsupported, "moddown: more than 16 dropped primes");
  const uint32_t *c1 = type == MDType::kModDown ? m.mod_down1.data()
                       : type == MDType::kRescale ? m.rs1.data() : m.mdr1.data();
  const int32_t *table = type == MDType::kModDown ? m.d_mod_down2 : type == MDType::kRescale ? m.d_rs2 : m.d_mdr2;
  const uint32_t *inv = type == MDType::kModDown ? m.inv_p_prod.data()
                        : type == MDType::kRescale ? m.rs_inv.data() : m.mdr_inv.data();
  const uint32_t *pad = type == MDType::kModDown ? nullptr
                        : type == MDType::kRescale ? m.rs_pad.data() : m.mdr_pad.data();
  std::vector<int> gs(ns.total()), gd(nd.total());
  P->gidx(ns, gs.data());
  P->gidx(nd, gd.data());
  std::vector<int> srows;
  const bool on_main = ns.main > nn.main, on_ter = ns.ter > nn.ter;
  CHD_CHECK(!(on_main && on_ter), kErrInvalidArg, "moddown: invalid prime combination");
  if (!on_ter)
    for (int r = ns.ter + nn.main; r < ns.q(); r++) srows.push_back(r);
  else
    for (int r = 0; r < ns.ter - nn.ter; r++) srows.push_back(r);
  for (int a = 0; a < nsa; a++) srows.push_back(ns.q() + a);
  CHD_CHECK(static_cast<int>(srows.size()) == src_len, kErrInvalidArg, "moddown: internal row mismatch");
  HeldScope scope(arena, hold);
  int32_t *xt = static_cast<int32_t *>(arena.alloc(static_cast<size_t>(npoly) * src_len * n * 4));
  CHD_CHECK(xt, kErrAlloc, "moddown: scratch allocation failed");
  std::vector<RowDesc> rows;
  const bool fused = P->log_n == 16;
  for (int p = 0; p < npoly; p++)
    for (int i = 0; i < src_len; i++) {
      const int gg = gs[srows[i]];
      RowDesc d{};
      d.src = src[p] + static_cast<size_t>(srows[i]) * n;
      d.dst = reinterpret_cast<uint32_t *>(xt) + (static_cast<size_t>(p) * src_len + i) * n;
      d.tw = itw(gg);
      d.q = P->primes[gg];
      mont_as_shoup(c1[i], gg, &d.c0, &d.c0s);
      d.flags = kCentre;
      rows.push_back(d);
    }
  if (fused) {
    for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_inv_rows(rb, P->log_n, stream); });
    MSColBatch b{};
    b.engine = ks_engine;
    b.err = d_err;
    b.tw = d_tw;
    b.itw = d_itw;
    b.primes = d_primes;
    b.qinvs = d_qinv;
    for (int p = 0; p < npoly; p++) {
      MSColJob &j = b.jobs[b.count++];
      j.src = reinterpret_cast<uint32_t *>(xt) + static_cast<size_t>(p) * src_len * n;
      j.dst = dst[p];
      j.table = table;
      j.K = src_len;
      j.M = dst_len;
      for (int i = 0; i < src_len; i++) {
        const int gg = gs[srows[i]];
        j.src_row[i] = static_cast<uint8_t>(i);
        j.src_gidx[i] = static_cast<uint8_t>(gg);
        mont_as_shoup(c1[i], gg, &j.c0[i], &j.c0s[i]);
      }
      for (int y = 0; y < dst_len; y++) {
        j.dst_row[y] = static_cast<uint8_t>(y);
        j.dst_gidx[y] = static_cast<uint8_t>(gd[y]);
      }
      if (b.count == kMaxMSColJobs) {
        launch_modswitch_cols(b, P->log_n, stream);
        b.count = 0;
      }
    }
    launch_modswitch_cols(b, P->log_n, stream);
  } else {
    for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_inv(rb, P->log_n, stream); });
    BConvBatch b{};
    b.primes = d_primes;
    b.qinvs = d_qinv;
    for (int p = 0; p < npoly; p++) {
      BConvJob &j = b.jobs[b.count++];
      j.xt = xt + static_cast<size_t>(p) * src_len * n;
      j.out = dst[p];
      j.table = table;
      j.K = src_len;
      j.M = dst_len;
      for (int y = 0; y < dst_len; y++) {
        j.out_row[y] = static_cast<uint8_t>(y);
        j.out_gidx[y] = static_cast<uint8_t>(gd[y]);
      }
      if (b.count == kMaxBConvJobs) {
        launch_bconv(b, P->log_n, stream);
        b.count = 0;
      }
    }
    launch_bconv(b, P->log_n, stream);
  }
  const int src2_start = nd.ter - nn.ter, src2_end = src2_start + nn.q();
  const int src2_off = std::max(0, ns.ter - nd.ter);
  rows.clear();
  for (int p = 0; p < npoly; p++)
    for (int y = 0; y < dst_len; y++) {
      RowDesc d{};
      d.src = d.dst = dst[p] + static_cast<size_t>(y) * n;
      d.tw = tw(gd[y]);
      d.q = P->primes[gd[y]];
      mont_as_shoup(inv[y], gd[y], &d.c2, &d.c2s);
      d.flags = kModDownEpi;
      if (y >= src2_start && y < src2_end) {
        d.flags |= kHasSrc2;
        d.src2 = src[p] + static_cast<size_t>(src2_off + y - src2_start) * n;
        if (pad) {
          d.flags |= kPadSrc2;
          mont_as_shoup(pad[y - src2_start], gd[y], &d.c1, &d.c1s);
        }
      }
      rows.push_back(d);
    }
  if (fused)
    for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_fwd_rows(rb, P->log_n, stream); });
  else
    for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_fwd(rb, P->log_n, stream); });
  return check_cuda("moddown");
}

// --------------------------------------------------------- evaluator
Status Context::key_switch_core(int level, const uint32_t *d0, const uint32_t *d1, const uint32_t *d_in,
                                const DeviceEvk &key, uint32_t *acc_b, uint32_t *acc_a) {
  KSJob j{d0, d1, d_in, acc_b, acc_a};
  return key_switch_many(level, 1, &j, key);
}

Status Context::key_switch_many(int level, int count, const KSJob *jobs, const DeviceEvk &key) {
  // Context.cpp:609-712 (MultKeyNoModDown with the CAccum of P * (d0, d1))
  const LevelMS &m = lms(level);
  const int n = P->n;
  NP np = P->level_np(level, P->alpha);
  const int nq = np.q(), tot = np.total();
  CHD_CHECK(tot <= 64 && m.beta <= 8, kErrUnsupported, "key switch: more than 64 primes or 8 digits");
  CHD_CHECK(key.np.aux == P->alpha && key.np.q() == P->L, kErrKey, "key switch: key basis mismatch");
  const int prime_offset = P->max_ter - np.ter;
  ArenaScope scope(arena);
  const size_t mu_words = static_cast<size_t>(tot) * n;
  uint32_t *mu_all = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(count) * m.beta * mu_words * 4));
  CHD_CHECK(mu_all, kErrAlloc, "key switch: scratch allocation failed");
  std::vector<uint32_t *> mu_ptrs(static_cast<size_t>(count) * m.beta);
  std::vector<uint32_t *const *> dsts(count);
  std::vector<const uint32_t *> srcs(count);
  for (int c = 0; c < count; c++) {
    for (int i = 0; i < m.beta; i++) mu_ptrs[c * m.beta + i] = mu_all + (static_cast<size_t>(c) * m.beta + i) * mu_words;
    dsts[c] = mu_ptrs.data() + c * m.beta;
    srcs[c] = jobs[c].d_in;
  }
  CHD_TRY(modup_many(level, count, srcs.data(), dsts.data()));
  KeyMacDesc d{};
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  const size_t kstride = static_cast<size_t>(key.np.total()) * n;
  int nb = 0;
  std::vector<int> digits;
  for (int i = 0; i < m.beta; i++) {
    if (m.dig_e[i] <= 0) continue;
    CHD_CHECK(i < key.beta, kErrKey, "key switch: key has too few digits");
    d.kb[nb] = key.bx + i * kstride;
    d.ka[nb] = key.ax + i * kstride;
    digits.push_back(i);
    nb++;
  }
  d.beta = nb;
  d.rows = tot;
  d.nq = nq;
  for (int r = 0; r < tot; r++) {
    d.q[r] = P->primes[g[r]];
    d.qinv[r] = P->qinv[g[r]];
    d.key_row[r] = static_cast<int16_t>(r < nq ? prime_offset + r : P->L + (r - nq));
    d.p_prod[r] = r < nq ? p_prod[prime_offset + r] : 0;
  }
  for (int c0 = 0; c0 < count; c0 += kMaxKeyMacCts) {
    d.count = std::min(kMaxKeyMacCts, count - c0);
    for (int c = 0; c < d.count; c++) {
      const KSJob &j = jobs[c0 + c];
      KeyMacCt &k = d.ct[c];
      for (int b = 0; b < nb; b++) k.mu[b] = mu_ptrs[(c0 + c) * m.beta + digits[b]];
      k.d0 = j.d0;
      k.d1 = j.d1;
      k.acc_b = j.acc_b;
      k.acc_a = j.acc_a;
    }
    launch_key_mac(d, P->log_n, stream);
  }
  return check_cuda("key switch");
}

static int level_of(const Params &P, const DeviceCt &a) { return P.np_to_level(NP{a.np.main, a.np.ter, 0}); }

Status Context::hmult(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key, bool rescale) {
  // Context.cpp:862-871: Mult (tensor) then RelinearizeRescale (merged
  // ModDown+Rescale) or Relinearize
  CHD_CHECK(a.np == b.np && a.np.aux == 0, kErrShape, "HMult: operands must share a level and have no aux primes");
  CHD_CHECK(!a.has_rx && !b.has_rx, kErrShape, "Relinearization required before Mult Ct x Ct");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "HMult: invalid level");
  CHD_CHECK(!rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  const int n = P->n, nq = a.np.q(), tot = nq + P->alpha;
  CHD_CHECK(tot <= 64, kErrUnsupported, "HMult: more than 64 primes in the extended basis");
  if (n == 65536) {
    // fused pipeline; an aliased result is written through a scratch copy
    if (&res != &a && &res != &b) {
      DeviceCt *r[1] = {&res};
      const DeviceCt *x[1] = {&a}, *y[1] = {&b};
      return hmult_batch(1, r, x, y, key, rescale);
    }
    ArenaScope scope(arena);
    NP out_np = P->level_np(rescale ? level - 1 : level, 0);
    const size_t words = static_cast<size_t>(out_np.total()) * n;
    uint32_t *tb = static_cast<uint32_t *>(arena.alloc(words * 4)), *ta = static_cast<uint32_t *>(arena.alloc(words * 4));
    CHD_CHECK(tb && ta, kErrAlloc, "HMult: scratch allocation failed");
    KSIn in{0, a.bx, a.ax, b.bx, b.ax, tb, ta};
    const double sc = rescale ? a.scale * b.scale / P->rescale_prod[level] : a.scale * b.scale;
    const int slots = std::max(a.num_slots, b.num_slots);
    CHD_TRY(key_switch_fused(level, 1, &in, key, rescale ? MDType::kModDownRescale : MDType::kModDown));
    CHD_TRY(res.reserve(out_np, false, n));
    cudaMemcpyAsync(res.bx, tb, words * 4, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(res.ax, ta, words * 4, cudaMemcpyDeviceToDevice, stream);
    res.scale = sc;
    res.num_slots = slots;
    return check_cuda("hmult");
  }
  ArenaScope scope(arena);
  uint32_t *d = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(3) * nq * n * 4));
  uint32_t *acc = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(2) * tot * n * 4));
  CHD_CHECK(d && acc, kErrAlloc, "HMult: scratch allocation failed");
  uint32_t *d0 = d, *d1 = d + static_cast<size_t>(nq) * n, *d2 = d + static_cast<size_t>(2) * nq * n;
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  TensorBatch tb{};
  for (int r = 0; r < nq; r++) {
    TensorRow &t = tb.rows[tb.count++];
    const size_t o = static_cast<size_t>(r) * n;
    t.b1 = a.bx + o;
    t.a1 = a.ax + o;
    t.b2 = b.bx + o;
    t.a2 = b.ax + o;
    t.d0 = d0 + o;
    t.d1 = d1 + o;
    t.d2 = d2 + o;
    t.q = P->primes[g[r]];
    t.qinv = P->qinv[g[r]];
  }
  launch_tensor(tb, P->log_n, stream);
  uint32_t *acc_b = acc, *acc_a = acc + static_cast<size_t>(tot) * n;
  CHD_TRY(key_switch_core(level, d0, d1, d2, key, acc_b, acc_a));
  const double sa = a.scale, sb = b.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  NP out_np = P->level_np(rescale ? level - 1 : level, 0);
  CHD_TRY(res.reserve(out_np, false, n));
  const uint32_t *srcs[2] = {acc_b, acc_a};
  uint32_t *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, rescale ? MDType::kModDownRescale : MDType::kModDown, srcs, dsts, 2));
  res.scale = rescale ? sa * sb / P->rescale_prod[level] : sa * sb;
  res.num_slots = slots;
  return kOk;
}

Status Context::hmult_batch(int count, DeviceCt *const *res, const DeviceCt *const *a, const DeviceCt *const *b,
                            const DeviceEvk &key, bool rescale) {
  // Batched Context::HMult: every stage (tensor, ModUp, key MAC, merged
  // ModDown+Rescale) runs once for the whole batch.  At N = 2^16 the pairs
  // may sit at different levels (one pipeline over all of them); below it a
  // mixed batch runs one pipeline per level.  Results must not alias other
  // pairs' operands (such a batch runs one pair at a time).
  if (count <= 0) return kOk;
  bool uniform = true, aliased = false;
  for (int i = 0; i < count; i++) {
    CHD_CHECK(a[i]->np == b[i]->np && a[i]->np.aux == 0 && !a[i]->has_rx && !b[i]->has_rx, kErrShape,
              "HMult batch: each pair must share a level, no aux primes, no rx");
    uniform = uniform && a[i]->np == a[0]->np;
    for (int j = 0; j < count; j++)
      if (res[i] == a[j] || res[i] == b[j]) aliased = true;
  }
  if (aliased) {  // results overwrite operands of other pairs: one by one
    for (int i = 0; i < count; i++) CHD_TRY(hmult(*res[i], *a[i], *b[i], key, rescale));
    return kOk;
  }
  if (P->log_n == 16) {
    std::vector<KSIn> in(count);
    std::vector<int> levels(count);
    for (int c = 0; c < count; c++) {
      const int level = level_of(*P, *a[c]);
      CHD_CHECK(level >= 0, kErrInvalidLevel, "HMult: invalid level");
      CHD_CHECK(!rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
      CHD_CHECK(a[c]->np.q() + P->alpha <= 64, kErrUnsupported, "HMult: more than 64 primes in the extended basis");
      levels[c] = level;
      const double sa = a[c]->scale, sb = b[c]->scale;
      const int slots = std::max(a[c]->num_slots, b[c]->num_slots);
      in[c] = KSIn{0, a[c]->bx, a[c]->ax, b[c]->bx, b[c]->ax, nullptr, nullptr};
      CHD_TRY(res[c]->reserve(P->level_np(rescale ? level - 1 : level, 0), false, P->n));
      res[c]->scale = rescale ? sa * sb / P->rescale_prod[level] : sa * sb;
      res[c]->num_slots = slots;
      in[c].out_b = res[c]->bx;
      in[c].out_a = res[c]->ax;
    }
    return key_switch_fused_levels(levels.data(), count, in.data(), key,
                                   rescale ? MDType::kModDownRescale : MDType::kModDown);
  }
  if (!uniform) {
    // mixed levels: one batched pipeline per level, in level order
    std::map<int, std::vector<int>> by_level;
    for (int i = 0; i < count; i++) by_level[-level_of(*P, *a[i])].push_back(i);
    for (const auto &e : by_level) {
      std::vector<DeviceCt *> r;
      std::vector<const DeviceCt *> x, y;
      for (int i : e.second) {
        r.push_back(res[i]);
        x.push_back(a[i]);
        y.push_back(b[i]);
      }
      CHD_TRY(hmult_batch(static_cast<int>(r.size()), r.data(), x.data(), y.data(), key, rescale));
    }
    return kOk;
  }
  const int level = level_of(*P, *a[0]);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "HMult: invalid level");
  CHD_CHECK(!rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  const int n = P->n, nq = a[0]->np.q(), tot = nq + P->alpha;
  CHD_CHECK(tot <= 64, kErrUnsupported, "HMult: more than 64 primes in the extended basis");
  ArenaScope scope(arena);
  const size_t qw = static_cast<size_t>(nq) * n, tw_ = static_cast<size_t>(tot) * n;
  uint32_t *d = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(count) * 3 * qw * 4));
  uint32_t *acc = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(count) * 2 * tw_ * 4));
  CHD_CHECK(d && acc, kErrAlloc, "HMult: scratch allocation failed");
  std::vector<int> g(nq);
  P->gidx(a[0]->np, g.data());
  TensorBatch tb{};
  std::vector<KSJob> jobs(count);
  for (int c = 0; c < count; c++) {
    uint32_t *d0 = d + c * 3 * qw, *d1 = d0 + qw, *d2 = d1 + qw;
    for (int r = 0; r < nq; r++) {
      if (tb.count == 64) {
        launch_tensor(tb, P->log_n, stream);
        tb.count = 0;
      }
      TensorRow &t = tb.rows[tb.count++];
      const size_t o = static_cast<size_t>(r) * n;
      t.b1 = a[c]->bx + o;
      t.a1 = a[c]->ax + o;
      t.b2 = b[c]->bx + o;
      t.a2 = b[c]->ax + o;
      t.d0 = d0 + o;
      t.d1 = d1 + o;
      t.d2 = d2 + o;
      t.q = P->primes[g[r]];
      t.qinv = P->qinv[g[r]];
    }
    jobs[c] = KSJob{d0, d1, d2, acc + c * 2 * tw_, acc + c * 2 * tw_ + tw_};
  }
  launch_tensor(tb, P->log_n, stream);
  CHD_TRY(key_switch_many(level, count, jobs.data(), key));
  NP out_np = P->level_np(rescale ? level - 1 : level, 0);
  std::vector<const uint32_t *> srcs(2 * count);
  std::vector<uint32_t *> dsts(2 * count);
  for (int c = 0; c < count; c++) {
    const double sa = a[c]->scale, sb = b[c]->scale;
    const int slots = std::max(a[c]->num_slots, b[c]->num_slots);
    CHD_TRY(res[c]->reserve(out_np, false, n));
    res[c]->scale = rescale ? sa * sb / P->rescale_prod[level] : sa * sb;
    res[c]->num_slots = slots;
    srcs[2 * c] = jobs[c].acc_b;
    srcs[2 * c + 1] = jobs[c].acc_a;
    dsts[2 * c] = res[c]->bx;
    dsts[2 * c + 1] = res[c]->ax;
  }
  return moddown(level, rescale ? MDType::kModDownRescale : MDType::kModDown, srcs.data(), dsts.data(),
                 2 * count);
}

Status Context::relinearize(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key, bool rescale) {
  // Context.cpp:539-547 and :714-737
  CHD_CHECK(a.has_rx && a.np.aux == 0, kErrShape, "Relinearize requires a ciphertext with rx");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "Relinearize: invalid level");
  CHD_CHECK(!rescale || level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  const int n = P->n, tot = a.np.q() + P->alpha;
  if (n == 65536) {
    ArenaScope scope(arena);
    NP out_np = P->level_np(rescale ? level - 1 : level, 0);
    const size_t words = static_cast<size_t>(out_np.total()) * n;
    uint32_t *tb = static_cast<uint32_t *>(arena.alloc(words * 4)), *ta = static_cast<uint32_t *>(arena.alloc(words * 4));
    CHD_CHECK(tb && ta, kErrAlloc, "Relinearize: scratch allocation failed");
    KSIn in{2, a.bx, a.ax, nullptr, a.rx, tb, ta};
    const double sc = rescale ? a.scale / P->rescale_prod[level] : a.scale;
    const int slots = a.num_slots;
    CHD_TRY(key_switch_fused(level, 1, &in, key, rescale ? MDType::kModDownRescale : MDType::kModDown));
    CHD_TRY(res.reserve(out_np, false, n));
    cudaMemcpyAsync(res.bx, tb, words * 4, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(res.ax, ta, words * 4, cudaMemcpyDeviceToDevice, stream);
    res.scale = sc;
    res.num_slots = slots;
    return check_cuda("relinearize");
  }
  ArenaScope scope(arena);
  uint32_t *acc = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(2) * tot * n * 4));
  CHD_CHECK(acc, kErrAlloc, "Relinearize: scratch allocation failed");
  uint32_t *acc_b = acc, *acc_a = acc + static_cast<size_t>(tot) * n;
  CHD_TRY(key_switch_core(level, a.bx, a.ax, a.rx, key, acc_b, acc_a));
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(P->level_np(rescale ? level - 1 : level, 0), false, n));
  const uint32_t *srcs[2] = {acc_b, acc_a};
  uint32_t *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, rescale ? MDType::kModDownRescale : MDType::kModDown, srcs, dsts, 2));
  res.scale = rescale ? sc / P->rescale_prod[level] : sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::mult_key(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key) {
  // Context.cpp:584-607
  CHD_CHECK(!a.has_rx && a.np.aux == 0, kErrShape, "MultKey: ciphertext must be relinearised, no aux primes");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "MultKey: invalid level");
  const int n = P->n, tot = a.np.q() + P->alpha;
  if (n == 65536) {
    ArenaScope scope(arena);
    const size_t words = static_cast<size_t>(a.np.total()) * n;
    uint32_t *tb = static_cast<uint32_t *>(arena.alloc(words * 4)), *ta = static_cast<uint32_t *>(arena.alloc(words * 4));
    CHD_CHECK(tb && ta, kErrAlloc, "MultKey: scratch allocation failed");
    KSIn in{1, a.bx, a.ax, nullptr, nullptr, tb, ta};
    const double sc = a.scale;
    const int slots = a.num_slots;
    const NP np = a.np;
    CHD_TRY(key_switch_fused(level, 1, &in, key, MDType::kModDown));
    CHD_TRY(res.reserve(np, false, n));
    cudaMemcpyAsync(res.bx, tb, words * 4, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(res.ax, ta, words * 4, cudaMemcpyDeviceToDevice, stream);
    res.scale = sc;
    res.num_slots = slots;
    return check_cuda("mult key");
  }
  ArenaScope scope(arena);
  uint32_t *acc = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(2) * tot * n * 4));
  CHD_CHECK(acc, kErrAlloc, "MultKey: scratch allocation failed");
  uint32_t *acc_b = acc, *acc_a = acc + static_cast<size_t>(tot) * n;
  CHD_TRY(key_switch_core(level, a.bx, nullptr, a.ax, key, acc_b, acc_a));
  const double sc = a.scale;
  const int slots = a.num_slots;
  const NP np = a.np;
  CHD_TRY(res.reserve(np, false, n));
  const uint32_t *srcs[2] = {acc_b, acc_a};
  uint32_t *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, MDType::kModDown, srcs, dsts, 2));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::permute(DeviceCt &res, const DeviceCt &a, int amount) {
  // Context.cpp:501-527 (ElementWise.cu:370-391)
  CHD_CHECK(&res != &a, kErrInvalidArg, "Permute does not support in-place operation");
  CHD_CHECK(amount == -1 || (amount >= 0 && amount <= P->n / 2), kErrInvalidArg, "Permute: invalid amount");
  const int n = P->n, tot = a.np.total();
  CHD_TRY(res.reserve(a.np, a.has_rx, n));
  PermuteBatch pb{};
  pb.galois = P->galois_of(amount);
  std::vector<int> g(tot);
  P->gidx(a.np, g.data());
  const uint32_t *src[3] = {a.bx, a.ax, a.rx};
  uint32_t *dst[3] = {res.bx, res.ax, res.rx};
  const int parts = a.has_rx ? 3 : 2;
  for (int p = 0; p < parts; p++)
    for (int r = 0; r < tot; r++) {
      if (pb.count == kMaxPermuteRows) {
        launch_permute(pb, P->log_n, stream);
        pb.count = 0;
      }
      PermuteRow &pr = pb.rows[pb.count++];
      pr.src = src[p] + static_cast<size_t>(r) * n;
      pr.dst = dst[p] + static_cast<size_t>(r) * n;
      pr.add = nullptr;
      pr.src2 = nullptr;
      pr.q = P->primes[g[r]];
    }
  launch_permute(pb, P->log_n, stream);
  res.scale = a.scale;
  res.num_slots = a.num_slots;
  return check_cuda("permute");
}

// Temporary ciphertext carved from the arena (released with the enclosing
// ArenaScope; stream order makes the reuse safe).
Status scratch_ct(Arena &arena, DeviceCt &t, const NP &np, bool rx, int n) {
  const size_t words = static_cast<size_t>(np.total()) * n;
  t.owned = false;
  t.bx = static_cast<uint32_t *>(arena.alloc(words * 4));
  t.ax = static_cast<uint32_t *>(arena.alloc(words * 4));
  t.rx = rx ? static_cast<uint32_t *>(arena.alloc(words * 4)) : nullptr;
  t.cap_words = words;
  t.np = np;
  t.has_rx = rx;
  if (!t.bx || !t.ax || (rx && !t.rx)) {
    set_error("scratch allocation failed");
    return kErrAlloc;
  }
  return kOk;
}

Status Context::hrot(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key, int dist) {
  // Context.cpp:776-791: MultKey first, then the automorphism
  int slots = a.num_slots > 0 ? a.num_slots : P->n / 2;
  dist %= slots;
  if (dist < 0) dist += slots;
  if (dist == 0) {
    if (&res == &a) return kOk;
    const NP np = a.np;
    const bool rx = a.has_rx;
    CHD_TRY(res.reserve(np, rx, P->n));
    const size_t bytes = static_cast<size_t>(np.total()) * P->n * 4;
    cudaMemcpyAsync(res.bx, a.bx, bytes, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(res.ax, a.ax, bytes, cudaMemcpyDeviceToDevice, stream);
    if (rx) cudaMemcpyAsync(res.rx, a.rx, bytes, cudaMemcpyDeviceToDevice, stream);
    res.scale = a.scale;
    res.num_slots = a.num_slots;
    return check_cuda("hrot copy");
  }
  ArenaScope scope(arena);
  DeviceCt tmp;
  CHD_TRY(scratch_ct(arena, tmp, a.np, false, P->n));
  CHD_TRY(mult_key(tmp, a, key));
  return permute(res, tmp, dist);
}

Status Context::hconj(DeviceCt &res, const DeviceCt &a, const DeviceEvk &key) {
  ArenaScope scope(arena);
  DeviceCt tmp;
  CHD_TRY(scratch_ct(arena, tmp, a.np, false, P->n));
  CHD_TRY(mult_key(tmp, a, key));
  return permute(res, tmp, -1);
}

Status Context::hrot_batch(int count, DeviceCt *const *res, const DeviceCt *const *a, const DeviceEvk &key,
                           int dist) {
  const DeviceCt &a0 = *a[0];
  int d = dist;
  if (d != -1) {
    const int slots = a0.num_slots > 0 ? a0.num_slots : P->n / 2;
    d %= slots;
    if (d < 0) d += slots;
  }
  if (P->log_n != 16 || count == 1 || d == 0) {
    for (int c = 0; c < count; c++) {
      if (dist == -1)
        CHD_TRY(hconj(*res[c], *a[c], key));
      else
        CHD_TRY(hrot(*res[c], *a[c], key, dist));
    }
    return kOk;
  }
  CHD_CHECK(!a0.has_rx && a0.np.aux == 0, kErrShape, "MultKey: ciphertext must be relinearised, no aux primes");
  const int level = level_of(*P, a0);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "MultKey: invalid level");
  ArenaScope scope(arena);
  std::vector<DeviceCt> tmp(count);
  std::vector<KSIn> ins(count);
  for (int c = 0; c < count; c++) {
    CHD_CHECK(a[c]->np == a0.np && !a[c]->has_rx, kErrShape, "HRot batch: ciphertexts at different levels");
    CHD_TRY(scratch_ct(arena, tmp[c], a0.np, false, P->n));
    ins[c] = KSIn{1, a[c]->bx, a[c]->ax, nullptr, nullptr, tmp[c].bx, tmp[c].ax};
  }
  CHD_TRY(key_switch_fused(level, count, ins.data(), key, MDType::kModDown));
  for (int c = 0; c < count; c++) {
    tmp[c].scale = a[c]->scale;
    tmp[c].num_slots = a[c]->num_slots;
    CHD_TRY(permute(*res[c], tmp[c], d));
  }
  return kOk;
}

Status Context::hrot_add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b, const DeviceEvk &key, int dist) {
  // Context.cpp:800-830: res = Permute(MultKey(a)) + b
  CHD_CHECK(a.np == b.np, kErrShape, "HRotAdd: level mismatch");
  ArenaScope scope(arena);
  DeviceCt tmp;
  CHD_TRY(scratch_ct(arena, tmp, a.np, false, P->n));
  CHD_TRY(hrot(tmp, a, key, dist));
  return add(res, tmp, b);
}

Status Context::moddown_ct(DeviceCt &res, const DeviceCt &a) {
  CHD_CHECK(a.np.aux == P->alpha, kErrShape, "ModDown: input must carry all aux primes");
  const int level = P->np_to_level(NP{a.np.main, a.np.ter, 0});
  CHD_CHECK(level >= 0, kErrInvalidLevel, "ModDown: invalid level");
  NP out{a.np.main, a.np.ter, 0};
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_CHECK(&res != &a, kErrInvalidArg, "ModDown does not support in-place operation");
  CHD_TRY(res.reserve(out, false, P->n));
  const uint32_t *srcs[2] = {a.bx, a.ax};
  uint32_t *dsts[2] = {res.bx, res.ax};
  CHD_TRY(moddown(level, MDType::kModDown, srcs, dsts, 2));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::moddown_batch(int count, DeviceCt *const *res, const DeviceCt *const *a) {
  // ModDown of several ciphertexts at one level through one pipeline: the
  // 2 * count polynomials share the column pass and the row launches
  CHD_CHECK(count >= 1, kErrInvalidArg, "ModDown: empty batch");
  const NP np = a[0]->np;
  CHD_CHECK(np.aux == P->alpha, kErrShape, "ModDown: input must carry all aux primes");
  const int level = P->np_to_level(NP{np.main, np.ter, 0});
  CHD_CHECK(level >= 0, kErrInvalidLevel, "ModDown: invalid level");
  std::vector<const uint32_t *> srcs;
  std::vector<uint32_t *> dsts;
  for (int c = 0; c < count; c++) {
    CHD_CHECK(a[c]->np == np && !a[c]->has_rx, kErrShape, "ModDown: batch members at different levels");
    for (int d = 0; d < count; d++)
      CHD_CHECK(res[c] != a[d], kErrInvalidArg, "ModDown does not support in-place operation");
    CHD_TRY(res[c]->reserve(NP{np.main, np.ter, 0}, false, P->n));
    srcs.push_back(a[c]->bx);
    srcs.push_back(a[c]->ax);
    dsts.push_back(res[c]->bx);
    dsts.push_back(res[c]->ax);
  }
  CHD_TRY(moddown(level, MDType::kModDown, srcs.data(), dsts.data(), 2 * count));
  for (int c = 0; c < count; c++) {
    res[c]->scale = a[c]->scale;
    res[c]->num_slots = a[c]->num_slots;
  }
  return kOk;
}

Status Context::hoisted_rotate(const DeviceCt &a, int R, const int *dists, const DeviceEvk *const *keys,
                               DeviceCt *const *out) {
  const DeviceCt *ap = &a;
  DeviceCt *const *op = out;
  return hoisted_rotate_batch(1, &ap, R, dists, keys, &op);
}

Status Context::hoisted_rotate_batch(int count, const DeviceCt *const *a, int R, const int *dists,
                                     const DeviceEvk *const *keys, DeviceCt *const *const *out) {
  // Hoist.cu:578-691 with the fused BS kernel of Hoist.cu:21-78: one ModUp
  // per ciphertext (all of them in one batched ModUp), then every rotation
  // of every ciphertext in one launch per kMaxHoistCts ciphertexts, results
  // left in Q u P
  CHD_CHECK(count >= 1, kErrInvalidArg, "hoisted rotate: empty batch");
  const DeviceCt &a0 = *a[0];
  CHD_CHECK(!a0.has_rx && a0.np.aux == 0, kErrShape, "hoisted rotate: input must be relinearised");
  const int level = level_of(*P, a0);
  CHD_CHECK(level >= 0, kErrInvalidLevel, "hoisted rotate: invalid level");
  for (int c = 0; c < count; c++)
    CHD_CHECK(a[c]->np == a0.np && !a[c]->has_rx, kErrShape, "hoisted rotate: batch members at different levels");
  const LevelMS &m = lms(level);
  const int n = P->n;
  NP np = P->level_np(level, P->alpha);
  const int nq = np.q(), tot = np.total();
  CHD_CHECK(tot <= 64 && m.beta <= 8, kErrUnsupported, "hoisted rotate: too many primes");
  const int prime_offset = P->max_ter - np.ter;
  ArenaScope scope(arena);
  std::vector<std::vector<uint32_t *>> mu(count, std::vector<uint32_t *>(m.beta, nullptr));
  std::vector<uint32_t *const *> mu_p(count);
  std::vector<uint32_t *> bxp(count);
  std::vector<const uint32_t *> src(count);
  for (int c = 0; c < count; c++) {
    for (int i = 0; i < m.beta; i++) {
      mu[c][i] = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(tot) * n * 4));
      CHD_CHECK(mu[c][i], kErrAlloc, "hoisted rotate: scratch allocation failed");
    }
    mu_p[c] = mu[c].data();
    bxp[c] = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(nq) * n * 4));
    CHD_CHECK(bxp[c], kErrAlloc, "hoisted rotate: scratch allocation failed");
    src[c] = a[c]->ax;
  }
  CHD_TRY(modup_many(level, count, src.data(), mu_p.data()));
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  {
    ElemBatch eb{};
    for (int c = 0; c < count; c++)
      for (int r = 0; r < nq; r++) {
        if (eb.count == kMaxElemRows) {
          launch_elementwise(ElemOp::kMultConst, eb, P->log_n, stream);
          eb.count = 0;
        }
        ElemRow &e = eb.rows[eb.count++];
        e.a = a[c]->bx + static_cast<size_t>(r) * n;
        e.dst = bxp[c] + static_cast<size_t>(r) * n;
        e.q = P->primes[g[r]];
        e.qinv = P->qinv[g[r]];
        e.k = p_prod[prime_offset + r];
      }
    launch_elementwise(ElemOp::kMultConst, eb, P->log_n, stream);
  }
  const int slots = a0.num_slots > 0 ? a0.num_slots : n / 2;
  std::vector<int> dd(R);
  for (int j = 0; j < R; j++) {
    dd[j] = dists[j] % slots;
    if (dd[j] < 0) dd[j] += slots;
    CHD_CHECK(dd[j] > 0 && dd[j] < n / 2, kErrInvalidArg, "hoisted rotate: invalid rotation");
    for (int c = 0; c < count; c++) {
      DeviceCt *o = out[c][j];
      CHD_TRY(o->reserve(np, false, n));
      o->scale = a[c]->scale;
      o->num_slots = a[c]->num_slots;
    }
  }
  const size_t kstride = static_cast<size_t>(P->L + P->alpha) * n;
  for (int j0 = 0; j0 < R; j0 += kMaxHoist) {
    for (int c0 = 0; c0 < count; c0 += kMaxHoistCts) {
      HoistDesc d{};
      d.count = std::min(kMaxHoistCts, count - c0);
      int nb = 0;
      for (int i = 0; i < m.beta; i++) {
        if (m.dig_e[i] <= 0) continue;
        for (int c = 0; c < d.count; c++) d.mu[c][nb] = mu[c0 + c][i];
        nb++;
      }
      for (int c = 0; c < d.count; c++) d.bxp[c] = bxp[c0 + c];
      d.beta = nb;
      d.rows = tot;
      d.nq = nq;
      d.R = std::min(kMaxHoist, R - j0);
      for (int r = 0; r < tot; r++) {
        d.q[r] = P->primes[g[r]];
        d.qinv[r] = P->qinv[g[r]];
        d.key_row[r] = static_cast<int16_t>(r < nq ? prime_offset + r : P->L + (r - nq));
      }
      for (int j = 0; j < d.R; j++) {
        const DeviceEvk &k = *keys[j0 + j];
        CHD_CHECK(k.np.aux == P->alpha && k.np.q() == P->L, kErrKey, "hoisted rotate: key basis mismatch");
        int b = 0;
        for (int i = 0; i < m.beta; i++) {
          if (m.dig_e[i] <= 0) continue;
          CHD_CHECK(i < k.beta, kErrKey, "hoisted rotate: key has too few digits");
          d.kb[j][b] = k.bx + i * kstride;
          d.ka[j][b] = k.ax + i * kstride;
          b++;
        }
        for (int c = 0; c < d.count; c++) {
          d.out_b[c][j] = out[c0 + c][j0 + j]->bx;
          d.out_a[c][j] = out[c0 + c][j0 + j]->ax;
        }
        d.galois_inv[j] = P->galois_of(n / 2 - dd[j0 + j]);
      }
      launch_hoisted(d, P->log_n, stream, ks_engine == 2);
    }
  }
  return check_cuda("hoisted rotate");
}

// ------------------------------------------------------- element-wise ops
// one element-wise op over `parts` parts of every row of np (row r of
// part p at dst[p] + r * N, likewise a / b), per-row constant k[r]
Status elem_parts(Context &C, ElemOp op, const NP &np, int parts, uint32_t *const *dst, const uint32_t *const *a,
                  const uint32_t *const *b, const uint32_t *k) {
  const int n = C.P->n, tot = np.total();
  std::vector<int> g(tot);
  C.P->gidx(np, g.data());
  ElemBatch eb{};
  for (int p = 0; p < parts; p++)
    for (int r = 0; r < tot; r++) {
      if (eb.count == kMaxElemRows) {
        launch_elementwise(op, eb, C.P->log_n, C.stream);
        eb.count = 0;
      }
      ElemRow &e = eb.rows[eb.count++];
      e.a = a[p] + static_cast<size_t>(r) * n;
      e.b = b ? b[p] + static_cast<size_t>(r) * n : nullptr;
      e.c = nullptr;
      e.dst = dst[p] + static_cast<size_t>(r) * n;
      e.q = C.P->primes[g[r]];
      e.qinv = C.P->qinv[g[r]];
      e.k = k ? k[r] : 0;
    }
  launch_elementwise(op, eb, C.P->log_n, C.stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

Status Context::add(DeviceCt &res, const DeviceCt &a, const DeviceCt &b) {
  // Context.cpp:145-172
  CHD_CHECK(a.np == b.np, kErrShape, "Add: level mismatch");
  const bool both_rx = a.has_rx && b.has_rx;
  const DeviceCt *rx_src = a.has_rx ? &a : (b.has_rx ? &b : nullptr);
  const uint32_t *keep_rx = (!both_rx && rx_src) ? rx_src->rx : nullptr;
  const bool out_rx = a.has_rx || b.has_rx;
  if ((&res == &a || &res == &b) && out_rx && !res.rx && res.owned) {
    // the result needs an rx buffer its aliased input lacks: growing it
    // would free the input before it is read
    DeviceCt tmp;
    CHD_TRY(add(tmp, a, b));
    res = std::move(tmp);
    return kOk;
  }
  const NP np = a.np;
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx}, *pb[3] = {b.bx, b.ax, b.rx};
  const double sc = a.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  CHD_TRY(res.reserve(np, out_rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kAdd, np, both_rx ? 3 : 2, pd, pa, pb, nullptr));
  if (keep_rx && keep_rx != res.rx)
    cudaMemcpyAsync(res.rx, keep_rx, static_cast<size_t>(np.total()) * P->n * 4, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::sub(DeviceCt &res, const DeviceCt &a, const DeviceCt &b) {
  // Context.cpp:205-229: with rx on one side only, res.rx = a.rx or -b.rx
  CHD_CHECK(a.np == b.np, kErrShape, "Sub: level mismatch");
  const bool both_rx = a.has_rx && b.has_rx;
  const bool out_rx = a.has_rx || b.has_rx;
  const uint32_t *only_rx = (!both_rx && out_rx) ? (a.has_rx ? a.rx : b.rx) : nullptr;
  const bool neg_rx = !both_rx && b.has_rx;
  if ((&res == &a || &res == &b) && out_rx && !res.rx && res.owned) {
    // the result needs an rx buffer its aliased input lacks: growing it
    // would free the input before it is read
    DeviceCt tmp;
    CHD_TRY(sub(tmp, a, b));
    res = std::move(tmp);
    return kOk;
  }
  const NP np = a.np;
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx}, *pb[3] = {b.bx, b.ax, b.rx};
  const double sc = a.scale;
  const int slots = std::max(a.num_slots, b.num_slots);
  CHD_TRY(res.reserve(np, out_rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kSub, np, both_rx ? 3 : 2, pd, pa, pb, nullptr));
  if (neg_rx) {
    const uint32_t *src[1] = {only_rx};
    uint32_t *dst[1] = {res.rx};
    CHD_TRY(elem_parts(*this, ElemOp::kNeg, np, 1, dst, src, nullptr, nullptr));
  } else if (only_rx && only_rx != res.rx) {
    cudaMemcpyAsync(res.rx, only_rx, static_cast<size_t>(np.total()) * P->n * 4, cudaMemcpyDeviceToDevice, stream);
  }
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::neg(DeviceCt &res, const DeviceCt &a) {
  const NP np = a.np;
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx};
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kNeg, np, rx ? 3 : 2, pd, pa, nullptr, nullptr));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::mult_tensor(DeviceCt &res, const DeviceCt &a, const DeviceCt &b) {
  // Context.cpp:316-330
  CHD_CHECK(a.np == b.np && a.np.aux == 0, kErrShape, "Mult: level mismatch");
  CHD_CHECK(!a.has_rx && !b.has_rx, kErrShape, "Relinearization required before Mult Ct x Ct");
  CHD_CHECK(&res != &a && &res != &b, kErrInvalidArg, "Mult: result must not alias an operand");
  const int n = P->n, nq = a.np.q();
  CHD_CHECK(nq <= 64, kErrUnsupported, "Mult: more than 64 primes");
  CHD_TRY(res.reserve(a.np, true, n));
  std::vector<int> g(nq);
  P->gidx(a.np, g.data());
  TensorBatch tb{};
  for (int r = 0; r < nq; r++) {
    TensorRow &t = tb.rows[tb.count++];
    const size_t o = static_cast<size_t>(r) * n;
    t.b1 = a.bx + o;
    t.a1 = a.ax + o;
    t.b2 = b.bx + o;
    t.a2 = b.ax + o;
    t.d0 = res.bx + o;
    t.d1 = res.ax + o;
    t.d2 = res.rx + o;
    t.q = P->primes[g[r]];
    t.qinv = P->qinv[g[r]];
  }
  launch_tensor(tb, P->log_n, stream);
  res.scale = a.scale * b.scale;
  res.num_slots = std::max(a.num_slots, b.num_slots);
  return check_cuda("mult");
}

Status Context::mult_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx, double cscale) {
  const NP np = a.np;
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx};
  const bool rx = a.has_rx;
  const double sc = a.scale * cscale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kMultConst, np, rx ? 3 : 2, pd, pa, nullptr, cx));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::add_const(DeviceCt &res, const DeviceCt &a, const uint32_t *cx) {
  const NP np = a.np;
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  const uint32_t *pa[1] = {a.bx};
  const uint32_t *keep[2] = {a.ax, a.rx};
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[1] = {res.bx};
  CHD_TRY(elem_parts(*this, ElemOp::kAddConst, np, 1, pd, pa, nullptr, cx));
  const size_t bytes = static_cast<size_t>(np.total()) * P->n * 4;
  if (keep[0] != res.ax) cudaMemcpyAsync(res.ax, keep[0], bytes, cudaMemcpyDeviceToDevice, stream);
  if (rx && keep[1] != res.rx) cudaMemcpyAsync(res.rx, keep[1], bytes, cudaMemcpyDeviceToDevice, stream);
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::mult_plain(DeviceCt &res, const DeviceCt &a, const uint32_t *pt, double pscale) {
  const NP np = a.np;
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx};
  const uint32_t *pp[3] = {pt, pt, pt};
  const bool rx = a.has_rx;
  const double sc = a.scale * pscale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kMult, np, rx ? 3 : 2, pd, pa, pp, nullptr));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::mult_imag_unit(DeviceCt &res, const DeviceCt &a) {
  // ElementWise.cu:625-658: multiply by X^(N/2) = +-psi^(N/2) (psi_rev[1])
  CHD_CHECK(a.np.aux == 0, kErrShape, "MultImaginaryUnit: no aux primes");
  const NP np = a.np;
  std::vector<int> g(np.total());
  P->gidx(np, g.data());
  std::vector<uint32_t> k(np.total());
  for (int r = 0; r < np.total(); r++) k[r] = imag_unit[g[r]];
  const uint32_t *pa[3] = {a.bx, a.ax, a.rx};
  const bool rx = a.has_rx;
  const double sc = a.scale;
  const int slots = a.num_slots;
  CHD_TRY(res.reserve(np, rx, P->n));
  uint32_t *pd[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(elem_parts(*this, ElemOp::kMultImagUnit, np, rx ? 3 : 2, pd, pa, nullptr, k.data()));
  res.scale = sc;
  res.num_slots = slots;
  return kOk;
}

Status Context::rescale(DeviceCt &res, const DeviceCt &a) {
  // Context.cpp:739-774
  CHD_CHECK(a.np.aux == 0, kErrShape, "Rescale is not supported for ciphertexts with p primes");
  CHD_CHECK(&res != &a, kErrInvalidArg, "Rescale does not support in-place operation");
  const int level = level_of(*P, a);
  CHD_CHECK(level >= 1, kErrInvalidLevel, "Not enough q primes to rescale");
  const bool rx = a.has_rx;
  CHD_TRY(res.reserve(P->level_np(level - 1, 0), rx, P->n));
  const uint32_t *srcs[3] = {a.bx, a.ax, a.rx};
  uint32_t *dsts[3] = {res.bx, res.ax, res.rx};
  CHD_TRY(moddown(level, MDType::kRescale, srcs, dsts, rx ? 3 : 2));
  res.scale = a.scale / P->rescale_prod[level];
  res.num_slots = a.num_slots;
  return kOk;
}

}  // namespace chd
