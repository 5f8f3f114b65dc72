"""Polynomial evaluation and EvalMod (src/extension/EvalPoly.cpp,
src/extension/EvalMod.cpp) compiled to op programs: the GPU run is
bit-exact with the oracle running the same program on its own primitives;
the program evaluated on plain values equals the polynomial (the compile
logic: split tree, Chebyshev fold-back, basis products, lazy rescaling); the
decrypted GPU result matches the plain value."""
import numpy as np
import pytest
from numpy.polynomial import chebyshev as cheb

import cheddar_b200 as chd
from boot_oracle import Ct, plain_program, run_program
from gpu_common import mult_key, pair, secret

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _encrypt(o, level, scale, msg, seed):
    # encryption of msg at exactly `scale` (the scale the program expects)
    pt = o.encode(level, scale, msg)
    return o.encrypt(seed, secret(KS), level, pt)


def _keys(g):
    (kb, ka), k = mult_key(KS)
    m = chd.EvkMap(g)
    m.set_mult(k)
    return m, (kb, ka)


def _coeffs(kind, degree, seed):
    rng = np.random.default_rng(seed)
    c = rng.random(degree + 1) * 2 - 1
    c /= np.arange(1, degree + 2) ** 1.5
    if kind == "even":
        c[1::2] = 0
    elif kind == "odd":
        c[0::2] = 0
    return c


@pytest.mark.parametrize("kind,degree", [("normal", 7), ("even", 14), ("odd", 15), ("normal", 31)])
def test_poly_program(cuda_ok, kind, degree):
    o, g = pair(KS)
    level = 20
    coeffs = _coeffs(kind, degree, degree)
    in_scale = o.rescale_prime_prod(level)
    target = 2.0 ** 30
    prog = chd.Program.poly(g, coeffs, level, in_scale, target, chebyshev=True)
    pj = prog.json()
    xs = np.linspace(-1, 1, 41)
    assert np.allclose(plain_program(pj, xs), cheb.chebval(xs, coeffs), rtol=0, atol=1e-12)
    keys, host_key = _keys(g)
    rng = np.random.default_rng(5)
    msg = rng.random(o.n // 2) * 2 - 1 + 0j
    bx, ax = _encrypt(o, level, in_scale, msg, 17)
    res = prog.run(g.import_ct(level, [bx, ax], in_scale), keys)
    ref = run_program(o, pj, Ct(level, [bx, ax], in_scale), mult_key=host_key)
    parts = res.numpy()
    assert len(parts) == 2 and len(ref.parts) == 2
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
    info = res.info()
    assert abs(info["scale"] - target) <= 1e-9 * target
    dec = o.decode(ref.level, target, o.decrypt(secret(KS), ref.level, parts), o.n // 2)
    assert np.abs(dec.real - cheb.chebval(msg.real, coeffs)).max() < 1e-3


def test_evalmod_program(cuda_ok):
    o, g = pair(KS)
    start = 20
    coeffs = chd.boot_mod_coefficients()
    prog = chd.Program.evalmod(g, start, coeffs, num_double_angle=3, initial_K=2)
    pj = prog.json()
    # plain: x = (I + e) / K  ->  sin(2 pi e) / (2 pi), the reference's
    # mod-1 approximation, for |I| < K
    K = 16
    rng = np.random.default_rng(3)
    I = rng.integers(-12, 13, 200)
    e = (rng.random(200) * 2 - 1) * 0.02
    x = (I + e) / K
    f = plain_program(pj, x)
    err = np.abs(f - np.sin(2 * np.pi * e) / (2 * np.pi)).max()
    assert err < 1e-5, err
    keys, host_key = _keys(g)
    msg = x[np.arange(o.n // 2) % len(x)] + 0j
    bx, ax = _encrypt(o, start, prog.start_scale, msg, 23)
    res = prog.run(g.import_ct(start, [bx, ax], prog.start_scale), keys)
    ref = run_program(o, pj, Ct(start, [bx, ax], prog.start_scale), mult_key=host_key)
    parts = res.numpy()
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
    assert ref.level == start - 8
    dec = o.decode(ref.level, prog.end_scale, o.decrypt(secret(KS), ref.level, parts), o.n // 2)
    # this parameter set rescales by single ~30-bit primes, so the CKKS noise
    # (amplified by K = 16 inside EvalMod) stays at the 2^-8 level
    assert np.abs(dec.real - plain_program(pj, msg.real)).max() < 1e-2
