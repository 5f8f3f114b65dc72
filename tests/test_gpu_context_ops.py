"""The remaining public Context operations (src/core/Context.cpp): Copy,
MultUnsafe Ct x Ct and Ct x Const at a target level (reading past the
inputs' extra terminal primes), MadUnsafe, Permute / PermuteConjugate,
HConjAdd, LevelDown, MultKeyNoModDown and IsMultUnsafeCompatible, bit-exact
against the oracle on the key-switching set (N = 2^16) and the set with
terminal primes (N = 2^12)."""
import numpy as np
import pytest

import cheddar_b200 as chd
from boot_oracle import add_mod, mont_mul
from gpu_common import mult_key, pair, rot_key, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"
RAT = "rational_t4_m10_a6.json"


def _eq(gpu_ct, ref_parts):
    parts = gpu_ct.numpy()
    assert len(parts) == len(ref_parts)
    for x, y in zip(parts, ref_parts):
        assert np.array_equal(x, y)


def _front(o, lvl_from, lvl_to):
    return o.level_np(lvl_from)[1] - o.level_np(lvl_to)[1]


def _const_mult(o, parts, front, cx, cfront, lvl):
    qs = o.primes(lvl)
    nq = len(qs)
    return [np.stack([mont_mul(p[front + r], cx[cfront + r], int(qs[r])) for r in range(nq)]) for p in parts]


def test_copy(cuda_ok):
    o, g = pair(KS)
    a = uniform_parts(KS, 17, 11)
    ga = g.import_ct(17, a, 3.0)
    c = g.Copy(ga)
    _eq(c, a)
    assert c.info()["scale"] == 3.0


@pytest.mark.parametrize("name,log_n,la,lb,level", [(KS, None, 20, 20, -1), (KS, None, 20, 18, 15),
                                                    (RAT, 12, 9, 8, 3), (RAT, 12, 9, 9, 6)])
def test_mult_unsafe(cuda_ok, name, log_n, la, lb, level):
    o, g = pair(name, log_n)
    a = uniform_parts(name, la, 21, log_n=log_n)
    b = uniform_parts(name, lb, 22, log_n=log_n)
    tgt = min(la, lb) if level == -1 else level
    assert g.IsMultUnsafeCompatible(la, tgt) and g.IsMultUnsafeCompatible(lb, tgt)
    r = g.MultUnsafe(g.import_ct(la, a, 2.0), g.import_ct(lb, b, 3.0), level)
    nq = o.num_q(tgt)
    fa, fb = _front(o, la, tgt), _front(o, lb, tgt)
    ref = o.tensor(tgt, a[0][fa:fa + nq], a[1][fa:fa + nq], b[0][fb:fb + nq], b[1][fb:fb + nq])
    _eq(r, list(ref))
    assert r.info()["scale"] == 6.0


@pytest.mark.parametrize("name,log_n,la,lc,level", [(KS, None, 20, 16, -1), (KS, None, 12, 20, 12),
                                                    (RAT, 12, 9, 6, -1), (RAT, 12, 6, 9, 4)])
def test_mult_unsafe_const_and_mad(cuda_ok, name, log_n, la, lc, level):
    o, g = pair(name, log_n)
    tgt = min(la, lc) if level == -1 else level
    assert g.IsMultUnsafeCompatible(la, tgt) and g.IsMultUnsafeCompatible(lc, tgt)
    a = uniform_parts(name, la, 31, log_n=log_n)
    cs = o.scale(lc)
    cx = o.encode_const(lc, cs, 0.375)
    ga = g.import_ct(la, a, 5.0)
    r = g.MultUnsafeConst(ga, cx, lc, cs, level)
    ref = _const_mult(o, a, _front(o, la, tgt), cx, _front(o, lc, tgt), tgt)
    _eq(r, ref)
    assert abs(r.info()["scale"] - 5.0 * cs) <= 1e-9 * 5.0 * cs
    # MadUnsafe: res (at tgt, scale a * c) += a * c
    r0 = uniform_parts(name, tgt, 32, log_n=log_n)
    gr = g.import_ct(tgt, r0, 5.0 * cs)
    g.MadUnsafe(gr, ga, cx, lc, cs)
    qs = o.primes(tgt)
    _eq(gr, [np.stack([add_mod(x[i], y[i], int(qs[i])) for i in range(len(qs))]) for x, y in zip(ref, r0)])
    with pytest.raises(chd.CheddarError):
        g.MadUnsafe(g.import_ct(tgt, r0, 1.0), ga, cx, lc, cs)  # scale mismatch


@pytest.mark.parametrize("rot", [3, 1234, 32767])
def test_permute_after_mult_key(cuda_ok, rot):
    # HRot = MultKey then Permute (Context.cpp:776-791)
    o, g = pair(KS)
    (kb, ka), key = rot_key(KS, rot)
    a = uniform_parts(KS, 19, 41)
    mk = g.MultKey(g.import_ct(19, a), key)
    _eq(g.Permute(mk, rot), o.hrot(19, a, (kb, ka), rot))
    _eq(g.Permute(mk, 0), mk.numpy())


def test_permute_conjugate_and_hconj_add(cuda_ok):
    o, g = pair(KS)
    (kb, ka), key = rot_key(KS, -1)
    a = uniform_parts(KS, 18, 51)
    b = uniform_parts(KS, 18, 52)
    mk = g.MultKey(g.import_ct(18, a), key)
    hc = o.hconj(18, a, (kb, ka))
    _eq(g.PermuteConjugate(mk), hc)
    qs = o.primes(18)
    ref = [np.stack([add_mod(x[i], y[i], int(qs[i])) for i in range(len(qs))]) for x, y in zip(hc, b)]
    _eq(g.HConjAdd(g.import_ct(18, a), g.import_ct(18, b), key), ref)


@pytest.mark.parametrize("name,log_n,level,target", [(KS, None, 20, 16), (RAT, 12, 7, 2), (KS, None, 7, 7)])
def test_level_down(cuda_ok, name, log_n, level, target):
    o, g = pair(name, log_n)
    a = uniform_parts(name, level, 61, log_n=log_n)
    r = g.LevelDown(g.import_ct(level, a, o.scale(level)), target)
    x = [p.copy() for p in a]
    for i in range(level, target, -1):
        cx = o.encode_const(i, o.scale(i), 1.0)
        x = _const_mult(o, x, 0, cx, 0, i)
        x = list(o.rescale_ct(i, np.stack(x)))
    _eq(r, x)
    with pytest.raises(chd.CheddarError):
        g.LevelDown(g.import_ct(level, a), level + 1)


def test_level_down_above_encryption_level(cuda_ok):
    # level-down constants exist for levels 1 .. default encryption level
    # (7 in this set); above it the call is an error, not a crash
    o, g = pair(RAT, 12)
    a = uniform_parts(RAT, 9, 62, log_n=12)
    with pytest.raises(chd.CheddarError):
        g.LevelDown(g.import_ct(9, a), 3)


def test_mult_key_no_moddown(cuda_ok):
    # ModDown(MultKeyNoModDown(a x b)) = Relinearize(a x b)
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    lvl = 21
    a = uniform_parts(KS, lvl, 71)
    b = uniform_parts(KS, lvl, 72)
    t = g.Mult(g.import_ct(lvl, a), g.import_ct(lvl, b))
    acc = g.MultKeyNoModDown(t, key)
    assert acc.info()["num_aux"] == o.alpha and not acc.info()["has_rx"]
    _eq(g.ModDown(acc), o.hmult(lvl, a, b, (kb, ka), rescale=False))
    with pytest.raises(chd.CheddarError):
        g.MultKeyNoModDown(g.import_ct(lvl, a), key)  # no rx


@pytest.mark.parametrize("name,log_n", [(KS, None), (RAT, 12)])
def test_mult_unsafe_compatible(cuda_ok, name, log_n):
    o, g = pair(name, log_n)
    for l1 in range(o.max_level + 1):
        for l2 in range(o.max_level + 1):
            lo, hi = o.level_np(min(l1, l2)), o.level_np(max(l1, l2))
            want = l1 == l2 or (lo[0] <= hi[0] and lo[1] <= hi[1])
            assert g.IsMultUnsafeCompatible(l1, l2) == want
    with pytest.raises(chd.CheddarError):
        g.IsMultUnsafeCompatible(-1, 0)
