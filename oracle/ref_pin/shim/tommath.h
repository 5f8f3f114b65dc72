// Project-written stand-in for the part of libtommath's public API that the
// reference's src/core/BigInt_tommath.cpp calls (the reference's default
// bigint backend, CMakeLists.txt:73-79; the library version is not pinned
// there, and it is not installed here).  Test infrastructure only: the
// reference build behind the parity tests links it.
//
// Behaviour restated from libtommath's documented API:
//  * mp_set_double truncates toward zero (the fraction bits below 2^0 are
//    shifted out of the magnitude, then the sign is applied);
//  * mp_get_double sums the magnitude's 60-bit digits from the most
//    significant one down, d = d * 2^60 + digit (the 64-bit build's
//    MP_DIGIT_BIT), then applies the sign;
//  * mp_mod returns a value in [0, |b|) for b > 0;
//  * mp_get_u64 returns the low 64 bits of the magnitude.
#pragma once

#include <cstdint>

typedef int mp_err;
typedef int mp_ord;

#define MP_OKAY 0
#define MP_VAL (-3)
#define MP_LT (-1)
#define MP_EQ 0
#define MP_GT 1

struct mp_int {
  int neg;           // 1 when negative (never set for zero)
  int used;          // number of 32-bit digits in use
  int alloc;         // digits allocated
  uint32_t *dp;      // little-endian magnitude
};

#ifdef __cplusplus
extern "C" {
#endif

mp_err mp_init(mp_int *a);
mp_err mp_init_u64(mp_int *a, uint64_t b);
mp_err mp_init_copy(mp_int *a, const mp_int *b);
mp_err mp_copy(const mp_int *a, mp_int *b);
void mp_clear(mp_int *a);
mp_err mp_set_double(mp_int *a, double b);
uint64_t mp_get_u64(const mp_int *a);
double mp_get_double(const mp_int *a);
mp_err mp_neg(const mp_int *a, mp_int *b);
mp_err mp_add(const mp_int *a, const mp_int *b, mp_int *c);
mp_err mp_sub(const mp_int *a, const mp_int *b, mp_int *c);
mp_err mp_mul(const mp_int *a, const mp_int *b, mp_int *c);
mp_err mp_div_2(const mp_int *a, mp_int *b);
mp_err mp_mod(const mp_int *a, const mp_int *b, mp_int *c);
mp_ord mp_cmp(const mp_int *a, const mp_int *b);
const char *mp_error_to_string(mp_err code);

#ifdef __cplusplus
}
#endif

#define mp_isneg(a) ((a)->neg != 0)
