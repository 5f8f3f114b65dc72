"""CPU checks of the reference build's support code (no GPU needed):

* the reference driver library (oracle/_ref/libcheddar_ref.so, built from
  the reference's sources when the reference tree is present) exports every
  entry point oracle/refdrv.py binds;
* the libtommath stand-in that the reference's BigInt_tommath.cpp links
  (oracle/ref_pin/shim/tommath_shim.cpp) follows libtommath's documented
  semantics on random operands, checked against Python integers: truncation
  toward zero in mp_set_double, a non-negative mp_mod, mp_get_double as the
  fold of 60-bit digits from the most significant one down, signed add /
  sub / mul, halving and comparison.
"""
import ctypes as C
import math
import os
import random

import pytest

import refdrv

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM_SO = os.path.join(HERE, "..", "oracle", "_ref", "libcheddar_ref.so")


def test_reference_driver_exports():
    if not refdrv.available():
        pytest.skip("reference driver not built (needs the reference tree)")
    L = refdrv.lib()
    assert L.refx_key_index_mult() == -22222222
    assert L.refx_key_index_conj() == 11111111


class MpInt(C.Structure):
    _fields_ = [("neg", C.c_int), ("used", C.c_int), ("alloc", C.c_int), ("dp", C.POINTER(C.c_uint32))]


@pytest.fixture(scope="module")
def mp():
    if not os.path.exists(SHIM_SO):
        pytest.skip("reference driver not built (needs the reference tree)")
    L = C.CDLL(SHIM_SO)
    P = C.POINTER(MpInt)
    for name, args, res in [("mp_init", [P], C.c_int), ("mp_init_u64", [P, C.c_uint64], C.c_int),
                            ("mp_set_double", [P, C.c_double], C.c_int), ("mp_get_u64", [P], C.c_uint64),
                            ("mp_get_double", [P], C.c_double), ("mp_neg", [P, P], C.c_int),
                            ("mp_add", [P, P, P], C.c_int), ("mp_sub", [P, P, P], C.c_int),
                            ("mp_mul", [P, P, P], C.c_int), ("mp_div_2", [P, P], C.c_int),
                            ("mp_mod", [P, P, P], C.c_int), ("mp_cmp", [P, P], C.c_int),
                            ("mp_clear", [P], None), ("mp_copy", [P, P], C.c_int)]:
        f = getattr(L, name)
        f.argtypes, f.restype = args, res
    return L


def _new(L, v=0):
    m = MpInt()
    L.mp_init(C.byref(m))
    _set(L, m, v)
    return m


def _set(L, m, v):
    # build |v| from 32-bit pieces: v = sum d_i 2^(32 i)
    mag = abs(v)
    acc = MpInt()
    L.mp_init_u64(C.byref(acc), 0)
    shift = MpInt()
    L.mp_init_u64(C.byref(shift), 1)
    base = MpInt()
    L.mp_init_u64(C.byref(base), 1 << 32)
    while mag:
        d = MpInt()
        L.mp_init_u64(C.byref(d), mag & 0xFFFFFFFF)
        L.mp_mul(C.byref(d), C.byref(shift), C.byref(d))
        L.mp_add(C.byref(acc), C.byref(d), C.byref(acc))
        L.mp_mul(C.byref(shift), C.byref(base), C.byref(shift))
        mag >>= 32
    if v < 0:
        L.mp_neg(C.byref(acc), C.byref(acc))
    L.mp_copy(C.byref(acc), C.byref(m))


def _val(m):
    v = 0
    for i in range(m.used):
        v |= m.dp[i] << (32 * i)
    return -v if m.neg else v


def _fold60(v):
    mag = abs(v)
    digits = []
    while mag:
        digits.append(mag & ((1 << 60) - 1))
        mag >>= 60
    d = 0.0
    for x in reversed(digits):
        d = d * float(2 ** 60) + float(x)
    return -d if v < 0 else d


def test_tommath_stand_in_semantics(mp):
    L = mp
    rng = random.Random(5)
    for _ in range(300):
        a = rng.randrange(-(1 << 300), 1 << 300)
        b = rng.randrange(-(1 << 200), 1 << 200) or 1
        p = rng.randrange(2, 1 << 31)
        ma, mb, mr, mpp = _new(L, a), _new(L, b), _new(L, 0), _new(L, p)
        assert _val(ma) == a and _val(mb) == b
        for f, want in [(L.mp_add, a + b), (L.mp_sub, a - b), (L.mp_mul, a * b)]:
            f(C.byref(ma), C.byref(mb), C.byref(mr))
            assert _val(mr) == want
        L.mp_mod(C.byref(ma), C.byref(mpp), C.byref(mr))
        assert _val(mr) == a % p
        L.mp_mod(C.byref(ma), C.byref(mb), C.byref(mr)) if b > 0 else None
        if b > 0:
            assert _val(mr) == a % b
        assert L.mp_cmp(C.byref(ma), C.byref(mb)) == (a > b) - (a < b)
        if a >= 0:
            L.mp_div_2(C.byref(ma), C.byref(mr))
            assert _val(mr) == a >> 1
        assert L.mp_get_double(C.byref(ma)) == _fold60(a)
    for _ in range(2000):
        x = rng.uniform(-1, 1) * 2.0 ** rng.randrange(-5, 120)
        m = _new(L, 0)
        L.mp_set_double(C.byref(m), x)
        assert _val(m) == math.trunc(x)
    m = _new(L, (1 << 64) - 5)
    assert L.mp_get_u64(C.byref(m)) == (1 << 64) - 5
