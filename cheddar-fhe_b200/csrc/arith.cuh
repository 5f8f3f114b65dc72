// Device modular arithmetic for 31-bit NTT-friendly primes.
//
// Residues are stored canonical in [0, q).  Products use signed Montgomery
// reduction with R = 2^32 (the same number representation as the reference,
// include/common/Basic.cuh:80-260 of scale-snu/cheddar-fhe: every evaluation-
// domain residue x is held as x * R mod q).  The reduction below follows the
// published signed-Montgomery method (G. Seiler, "Faster AVX2 optimized NTT
// multiplication for Ring-LWE lattice cryptography", 2018): for |a| < q*2^31
//   m = lo(a) * q^-1 mod 2^32 (signed),  r = hi(a) - hi(m * q)  in (-q, q),
// and r = a * 2^-32 mod q.
#pragma once

#include <cstdint>

namespace chd {

struct Modulus {
  uint32_t q;
  int32_t qinv;  // q^-1 mod 2^32 as a signed word
};

__device__ __forceinline__ int32_t mont_reduce_lazy(int64_t a, uint32_t q, int32_t qinv) {
  int32_t lo = static_cast<int32_t>(static_cast<uint32_t>(static_cast<uint64_t>(a)));
  int32_t hi = static_cast<int32_t>(a >> 32);
  int32_t m = lo * qinv;
  return hi - __mulhi(m, static_cast<int32_t>(q));
}

// a * b * 2^-32 mod q in (-q, q) for |a * b| < q * 2^31
__device__ __forceinline__ int32_t mont_mul_lazy(int32_t a, int32_t b, uint32_t q, int32_t qinv) {
  int32_t lo = a * b;
  int32_t hi = __mulhi(a, b);
  int32_t m = lo * qinv;
  return hi - __mulhi(m, static_cast<int32_t>(q));
}

__device__ __forceinline__ uint32_t canon(int32_t r, uint32_t q) {
  return static_cast<uint32_t>(r < 0 ? r + static_cast<int32_t>(q) : r);
}

// canonical Montgomery product of canonical operands
__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t q, int32_t qinv) {
  return canon(mont_mul_lazy(static_cast<int32_t>(a), static_cast<int32_t>(b), q, qinv), q);
}

__device__ __forceinline__ uint32_t mont_reduce(int64_t a, uint32_t q, int32_t qinv) {
  return canon(mont_reduce_lazy(a, q, qinv), q);
}

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) {
  uint32_t r = a + b;
  return r >= q ? r - q : r;
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t q) {
  int32_t r = static_cast<int32_t>(a) - static_cast<int32_t>(b);
  return static_cast<uint32_t>(r < 0 ? r + static_cast<int32_t>(q) : r);
}

__device__ __forceinline__ uint32_t neg_mod(uint32_t a, uint32_t q) { return a ? q - a : 0u; }

// centred representative in [-(q-1)/2, (q-1)/2] of a canonical residue
__device__ __forceinline__ int32_t centre(uint32_t a, uint32_t q) {
  return a > (q >> 1) ? static_cast<int32_t>(a) - static_cast<int32_t>(q) : static_cast<int32_t>(a);
}

// ---- two Montgomery products for one reduction (unsigned Montgomery
// reduction, P. Montgomery 1985).  For canonical a_i, b_i < q < 2^31 the sum
// s = a1 b1 + a2 b2 < 2 q^2 < 2^63; with m = s (-q^-1) mod 2^32 the value
// s + m q (< 2^64) is divisible by 2^32 and (s + m q) / 2^32 < 2q, congruent
// to s 2^-32, i.e. to mont_mul(a1, b1) + mont_mul(a2, b2).  qneg = -q^-1
// mod 2^32 (the negated qinv).
__device__ __forceinline__ uint32_t mont_redc2(uint64_t s, uint32_t q, uint32_t qneg) {
  const uint32_t m = static_cast<uint32_t>(s) * qneg;
  return static_cast<uint32_t>((s + static_cast<uint64_t>(m) * q) >> 32);
}
// canonical mont_mul(a1, b1) + mont_mul(a2, b2) for canonical operands
__device__ __forceinline__ uint32_t mont_mac2(uint32_t a1, uint32_t b1, uint32_t a2, uint32_t b2, uint32_t q,
                                              uint32_t qneg) {
  const uint64_t s = static_cast<uint64_t>(a1) * b1 + static_cast<uint64_t>(a2) * b2;
  const uint32_t r = mont_redc2(s, q, qneg);
  return r >= q ? r - q : r;
}

// Cooley-Tukey butterfly on canonical values: (a, b) -> (a + w b, a - w b)
__device__ __forceinline__ void ct_bfly(uint32_t &a, uint32_t &b, uint32_t w, uint32_t q, int32_t qinv) {
  uint32_t t = mont_mul(b, w, q, qinv);
  b = sub_mod(a, t, q);
  a = add_mod(a, t, q);
}

// Gentleman-Sande butterfly on canonical values: (a, b) -> (a + b, (a - b) w)
__device__ __forceinline__ void gs_bfly(uint32_t &a, uint32_t &b, uint32_t w, uint32_t q, int32_t qinv) {
  uint32_t d = sub_mod(a, b, q);
  a = add_mod(a, b, q);
  b = mont_mul(d, w, q, qinv);
}

// ---- Shoup multiplication with lazy [0, 2q) values (D. Harvey, "Faster
// arithmetic for number-theoretic transforms", 2014): for any 32-bit b and a
// constant w < q with companion ws = floor(w 2^32 / q),
//   b w - floor(b ws / 2^32) q  lies in [0, 2q)  (q < 2^31 keeps 2q in a word).
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t b, uint32_t w, uint32_t ws, uint32_t q) {
  return b * w - __umulhi(b, ws) * q;
}
// [0, 2q) -> [0, q): unsigned min(x, x - q)
__device__ __forceinline__ uint32_t reduce2q(uint32_t x, uint32_t q) { return min(x, x - q); }

// Cooley-Tukey butterfly, inputs and outputs in [0, 2q):
// (a, b) -> (a + w b, a - w b)
__device__ __forceinline__ void ct_lazy(uint32_t &a, uint32_t &b, uint2 w, uint32_t q) {
  const uint32_t x = reduce2q(a, q);
  const uint32_t t = reduce2q(shoup_lazy(b, w.x, w.y, q), q);
  a = x + t;
  b = x - t + q;
}
// Gentleman-Sande butterfly, inputs and outputs in [0, 2q):
// (a, b) -> (a + b, (a - b) w)
__device__ __forceinline__ void gs_lazy(uint32_t &a, uint32_t &b, uint2 w, uint32_t q) {
  const uint32_t x = reduce2q(a, q), y = reduce2q(b, q);
  a = x + y;
  b = shoup_lazy(x - y + q, w.x, w.y, q);
}

}  // namespace chd
