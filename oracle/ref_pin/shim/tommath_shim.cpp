// Implementation of the libtommath stand-in declared in tommath.h (same
// folder): sign-magnitude integers on 32-bit digits.  Test infrastructure.
#include "tommath.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

using Mag = std::vector<uint32_t>;

Mag get_mag(const mp_int *a) { return Mag(a->dp, a->dp + a->used); }

void trim(Mag &m) {
  while (!m.empty() && m.back() == 0) m.pop_back();
}

void put(mp_int *a, Mag m, int neg) {
  trim(m);
  if ((int)m.size() > a->alloc) {
    std::free(a->dp);
    a->alloc = (int)m.size() + 4;
    a->dp = static_cast<uint32_t *>(std::calloc(a->alloc, sizeof(uint32_t)));
  }
  if (!m.empty()) std::memcpy(a->dp, m.data(), m.size() * sizeof(uint32_t));
  a->used = (int)m.size();
  a->neg = m.empty() ? 0 : neg;
}

int cmp_mag(const Mag &a, const Mag &b) {
  if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
  for (size_t i = a.size(); i-- > 0;) {
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  }
  return 0;
}

Mag add_mag(const Mag &a, const Mag &b) {
  Mag r(std::max(a.size(), b.size()) + 1, 0);
  uint64_t c = 0;
  for (size_t i = 0; i < r.size(); ++i) {
    uint64_t s = c;
    if (i < a.size()) s += a[i];
    if (i < b.size()) s += b[i];
    r[i] = (uint32_t)s;
    c = s >> 32;
  }
  trim(r);
  return r;
}

// |a| >= |b| required.
Mag sub_mag(const Mag &a, const Mag &b) {
  Mag r(a.size(), 0);
  int64_t br = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    int64_t d = (int64_t)a[i] - br - (i < b.size() ? (int64_t)b[i] : 0);
    br = d < 0;
    r[i] = (uint32_t)(d + (br ? (int64_t)1 << 32 : 0));
  }
  trim(r);
  return r;
}

Mag mul_mag(const Mag &a, const Mag &b) {
  if (a.empty() || b.empty()) return Mag();
  Mag r(a.size() + b.size(), 0);
  for (size_t i = 0; i < a.size(); ++i) {
    uint64_t c = 0;
    for (size_t j = 0; j < b.size(); ++j) {
      uint64_t t = (uint64_t)a[i] * b[j] + r[i + j] + c;
      r[i + j] = (uint32_t)t;
      c = t >> 32;
    }
    size_t k = i + b.size();
    while (c != 0) {
      uint64_t t = (uint64_t)r[k] + c;
      r[k] = (uint32_t)t;
      c = t >> 32;
      ++k;
    }
  }
  trim(r);
  return r;
}

size_t bit_length(const Mag &m) {
  if (m.empty()) return 0;
  uint32_t top = m.back();
  size_t bits = 0;
  while (top) {
    ++bits;
    top >>= 1;
  }
  return (m.size() - 1) * 32 + bits;
}

Mag shl_mag(const Mag &m, size_t s) {
  if (m.empty()) return m;
  size_t w = s / 32, b = s % 32;
  Mag r(m.size() + w + 1, 0);
  for (size_t i = 0; i < m.size(); ++i) {
    uint64_t v = (uint64_t)m[i] << b;
    r[i + w] |= (uint32_t)v;
    r[i + w + 1] |= (uint32_t)(v >> 32);
  }
  trim(r);
  return r;
}

// Magnitude remainder |a| mod |b| (b nonzero).
Mag mod_mag(const Mag &a, const Mag &b) {
  if (b.size() == 1) {
    uint64_t d = b[0], r = 0;
    for (size_t i = a.size(); i-- > 0;) r = ((r << 32) | a[i]) % d;
    Mag out;
    if (r) out.push_back((uint32_t)r);
    return out;
  }
  Mag r = a;
  if (cmp_mag(r, b) < 0) return r;
  size_t lb = bit_length(b);
  for (size_t s = bit_length(r) - lb + 1; s-- > 0;) {
    Mag t = shl_mag(b, s);
    if (cmp_mag(r, t) >= 0) r = sub_mag(r, t);
  }
  return r;
}

// Signed add of (a, an) and (b, bn) into c.
void signed_add(const Mag &a, int an, const Mag &b, int bn, mp_int *c) {
  if (an == bn) {
    put(c, add_mag(a, b), an);
    return;
  }
  int k = cmp_mag(a, b);
  if (k == 0) {
    put(c, Mag(), 0);
  } else if (k > 0) {
    put(c, sub_mag(a, b), an);
  } else {
    put(c, sub_mag(b, a), bn);
  }
}

}  // namespace

mp_err mp_init(mp_int *a) {
  a->neg = 0;
  a->used = 0;
  a->alloc = 4;
  a->dp = static_cast<uint32_t *>(std::calloc(a->alloc, sizeof(uint32_t)));
  return MP_OKAY;
}

mp_err mp_init_u64(mp_int *a, uint64_t b) {
  mp_init(a);
  Mag m{(uint32_t)b, (uint32_t)(b >> 32)};
  put(a, m, 0);
  return MP_OKAY;
}

mp_err mp_init_copy(mp_int *a, const mp_int *b) {
  mp_init(a);
  return mp_copy(b, a);
}

mp_err mp_copy(const mp_int *a, mp_int *b) {
  if (a == b) return MP_OKAY;
  put(b, get_mag(a), a->neg);
  return MP_OKAY;
}

void mp_clear(mp_int *a) {
  std::free(a->dp);
  a->dp = nullptr;
  a->used = a->alloc = 0;
  a->neg = 0;
}

mp_err mp_set_double(mp_int *a, double b) {
  if (!std::isfinite(b)) return MP_VAL;
  double t = std::trunc(std::fabs(b));
  Mag m;
  if (t >= 1.0) {
    int e = 0;
    double f = std::frexp(t, &e);  // t = f * 2^e, f in [0.5, 1)
    uint64_t frac = (uint64_t)std::ldexp(f, 53);  // exact: 53 significant bits
    int shift = e - 53;
    Mag base{(uint32_t)frac, (uint32_t)(frac >> 32)};
    trim(base);
    if (shift >= 0) {
      m = shl_mag(base, (size_t)shift);
    } else {
      uint64_t v = frac >> (-shift);
      m = Mag{(uint32_t)v, (uint32_t)(v >> 32)};
    }
  }
  put(a, m, b < 0 ? 1 : 0);
  return MP_OKAY;
}

uint64_t mp_get_u64(const mp_int *a) {
  uint64_t lo = a->used > 0 ? a->dp[0] : 0;
  uint64_t hi = a->used > 1 ? a->dp[1] : 0;
  return lo | (hi << 32);
}

double mp_get_double(const mp_int *a) {
  // Regroup the magnitude into 60-bit digits, then fold from the top.
  Mag m = get_mag(a);
  size_t bits = bit_length(m);
  size_t ndig = (bits + 59) / 60;
  double d = 0.0;
  const double fac = std::ldexp(1.0, 60);
  for (size_t i = ndig; i-- > 0;) {
    uint64_t dig = 0;
    for (int k = 0; k < 60; ++k) {
      size_t bit = i * 60 + k;
      if (bit / 32 < m.size() && ((m[bit / 32] >> (bit % 32)) & 1u)) dig |= (uint64_t)1 << k;
    }
    d = d * fac + (double)dig;
  }
  return a->neg ? -d : d;
}

mp_err mp_neg(const mp_int *a, mp_int *b) {
  Mag m = get_mag(a);
  put(b, m, m.empty() ? 0 : !a->neg);
  return MP_OKAY;
}

mp_err mp_add(const mp_int *a, const mp_int *b, mp_int *c) {
  signed_add(get_mag(a), a->neg, get_mag(b), b->neg, c);
  return MP_OKAY;
}

mp_err mp_sub(const mp_int *a, const mp_int *b, mp_int *c) {
  signed_add(get_mag(a), a->neg, get_mag(b), !b->neg, c);
  return MP_OKAY;
}

mp_err mp_mul(const mp_int *a, const mp_int *b, mp_int *c) {
  put(c, mul_mag(get_mag(a), get_mag(b)), a->neg ^ b->neg);
  return MP_OKAY;
}

mp_err mp_div_2(const mp_int *a, mp_int *b) {
  Mag m = get_mag(a);
  for (size_t i = 0; i < m.size(); ++i) {
    m[i] = (m[i] >> 1) | (i + 1 < m.size() ? (m[i + 1] << 31) : 0u);
  }
  put(b, m, a->neg);
  return MP_OKAY;
}

mp_err mp_mod(const mp_int *a, const mp_int *b, mp_int *c) {
  Mag bm = get_mag(b);
  if (bm.empty()) return MP_VAL;
  Mag r = mod_mag(get_mag(a), bm);
  if (a->neg && !r.empty()) r = sub_mag(bm, r);
  put(c, r, 0);
  return MP_OKAY;
}

mp_ord mp_cmp(const mp_int *a, const mp_int *b) {
  if (a->neg != b->neg) return a->neg ? MP_LT : MP_GT;
  int k = cmp_mag(get_mag(a), get_mag(b));
  if (a->neg) k = -k;
  return k < 0 ? MP_LT : (k > 0 ? MP_GT : MP_EQ);
}

const char *mp_error_to_string(mp_err code) {
  return code == MP_OKAY ? "Successful" : "Value out of range";
}
