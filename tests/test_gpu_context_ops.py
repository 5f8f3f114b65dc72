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
        g.MultKeyNoModDown(g.import_ct(lvl, uniform_parts(KS, lvl, 73, num_aux=2), num_aux=2), key)  # aux primes


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


def _i64(x):
    return np.asarray(x, dtype=np.int64)


def _sub(x, y, Q):
    return ((_i64(x) - _i64(y)) % Q).astype(np.uint32)


def _add(x, y, Q):
    return ((_i64(x) + _i64(y)) % Q).astype(np.uint32)


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint32).view(np.int32)).cuda()


@pytest.mark.parametrize("name,log_n,level,rx,aux", [(KS, None, 20, False, 0), (KS, None, 13, True, 0),
                                                     (KS, None, 18, False, 8), (RAT, 12, 9, True, 0)])
def test_plain_and_const_ops(cuda_ok, name, log_n, level, rx, aux):
    # Add / Sub / Mult with a plaintext, Sub with a constant, and the
    # reversed Sub(Pt, Ct) / Sub(Const, Ct) (Context.cpp:171-304, 333-343)
    o, g = pair(name, log_n)
    parts = uniform_parts(name, level, 81, nparts=3 if rx else 2, log_n=log_n, num_aux=aux)
    qs = o.primes(level, aux)
    Q = _i64(qs)[:, None]
    pt = o.uniform(90, level, num_aux=aux)
    ptd = _dev(pt)
    sc = 2.0 ** 40
    ga = g.import_ct(level, parts, sc, num_aux=aux)
    _eq(g.AddPlain(ga, ptd, sc), [_add(parts[0], pt, Q)] + parts[1:])
    _eq(g.SubPlain(ga, ptd, sc), [_sub(parts[0], pt, Q)] + parts[1:])
    neg = [_sub(0, p, Q) for p in parts[1:]]
    _eq(g.SubPlainCt(ptd, sc, ga), [_sub(pt, parts[0], Q)] + neg)
    pr = g.MultPlain(ga, ptd, 3.0)
    _eq(pr, [np.stack([mont_mul(p[r], pt[r], int(qs[r])) for r in range(len(qs))]) for p in parts])
    assert pr.info()["scale"] == sc * 3.0
    cx = o.encode_const(level, sc, -0.625, num_aux=aux)
    C = _i64(cx)[:, None]
    _eq(g.SubConst(ga, cx), [_sub(parts[0], C, Q)] + parts[1:])
    _eq(g.SubConstCt(cx, sc, ga), [_sub(C, parts[0], Q)] + neg)
    with pytest.raises(chd.CheddarError):
        g.AddPlain(ga, ptd, sc * 2)  # scale mismatch
    with pytest.raises(chd.CheddarError):
        g.SubConstCt(cx, sc * (1 + 1e-9), ga)
    # in place: res aliases the ciphertext operand
    gi = g.import_ct(level, parts, sc, num_aux=aux)
    g.SubPlainCt(ptd, sc, gi, res=gi)
    _eq(gi, [_sub(pt, parts[0], Q)] + neg)


@pytest.mark.parametrize("name,log_n,la,a_aux,lp,p_aux,level", [
    (KS, None, 20, 0, 18, 0, -1), (KS, None, 20, 8, 20, 8, -1), (KS, None, 20, 8, 20, 0, -1),
    (KS, None, 19, 0, 21, 0, 12), (RAT, 12, 9, 0, 8, 0, -1), (RAT, 12, 9, 0, 9, 0, 6), (RAT, 12, 8, 0, 9, 0, 3)])
def test_mult_unsafe_plain(cuda_ok, name, log_n, la, a_aux, lp, p_aux, level):
    o, g = pair(name, log_n)
    tgt = min(la, lp) if level == -1 else level
    aux = min(a_aux, p_aux)
    a = uniform_parts(name, la, 101, log_n=log_n, num_aux=a_aux)
    pt = o.uniform(102, lp, num_aux=p_aux)
    qs = o.primes(tgt, aux)
    fa, fp = _front(o, la, tgt), _front(o, lp, tgt)
    ref = [np.stack([mont_mul(p[fa + r], pt[fp + r], int(qs[r])) for r in range(len(qs))]) for p in a]
    ga = g.import_ct(la, a, 2.0, num_aux=a_aux)
    r = g.MultUnsafePlain(ga, _dev(pt), lp, 5.0, pt_num_aux=p_aux, level=level)
    _eq(r, ref)
    info = r.info()
    assert info["num_aux"] == aux and info["scale"] == 10.0
    # in place with a level change goes through a temporary
    g.MultUnsafePlain(ga, _dev(pt), lp, 5.0, pt_num_aux=p_aux, level=level, res=ga)
    _eq(ga, ref)


@pytest.mark.parametrize("rot", [5, -1])
def test_mult_key_no_moddown_rotation(cuda_ok, rot):
    # without rx: ModUp(ax) (.) key + (P * bx, 0); ModDown of it = MultKey
    o, g = pair(KS)
    _, key = rot_key(KS, rot)
    a = uniform_parts(KS, 17, 111)
    ga = g.import_ct(17, a)
    acc = g.MultKeyNoModDown(ga, key)
    assert acc.info()["num_aux"] == o.alpha
    _eq(g.ModDown(acc), g.MultKey(ga, key).numpy())


def test_add_sub_mixed_rx(cuda_ok):
    # Context.cpp:146-229: with rx on one side only, res.rx = a.rx, or b.rx /
    # -b.rx; the result may alias the operand without rx
    o, g = pair(KS)
    lvl = 16
    Q = _i64(o.primes(lvl))[:, None]
    x = uniform_parts(KS, lvl, 121, nparts=3)
    y = uniform_parts(KS, lvl, 124)
    gx, gy = g.import_ct(lvl, x), g.import_ct(lvl, y)
    _eq(g.Add(gx, gy), [_add(x[0], y[0], Q), _add(x[1], y[1], Q), x[2]])
    _eq(g.Add(gy, gx), [_add(y[0], x[0], Q), _add(y[1], x[1], Q), x[2]])
    _eq(g.Sub(gx, gy), [_sub(x[0], y[0], Q), _sub(x[1], y[1], Q), x[2]])
    _eq(g.Sub(gy, gx), [_sub(y[0], x[0], Q), _sub(y[1], x[1], Q), _sub(0, x[2], Q)])
    g.Add(gx, gy, res=gy)
    _eq(gy, [_add(x[0], y[0], Q), _add(x[1], y[1], Q), x[2]])
    gy = g.import_ct(lvl, y)
    g.Sub(gy, gx, res=gy)
    _eq(gy, [_sub(y[0], x[0], Q), _sub(y[1], x[1], Q), _sub(0, x[2], Q)])


def test_misaligned_device_buffers_rejected(cuda_ok):
    # the kernels move device data in 16-byte vectors: a buffer that does
    # not start on a 16-byte boundary is an argument error, not a launch
    import torch
    o, g = pair(KS)
    lvl = 3
    rows = o.num_q(lvl)
    buf = torch.zeros(2, rows * o.n + 4, dtype=torch.int32, device="cuda")
    with pytest.raises(chd.CheddarError) as e:
        g.wrap_ct(lvl, [buf[0][1:], buf[1][1:]])
    assert e.value.code == 1
    ga = g.import_ct(lvl, uniform_parts(KS, lvl, 131))
    pt = torch.zeros(rows * o.n + 4, dtype=torch.int32, device="cuda")
    with pytest.raises(chd.CheddarError):
        g.MultPlain(ga, pt[2:], 1.0)
    with pytest.raises(chd.CheddarError):
        g.AddPlain(ga, pt[1:], 1.0)
    # aligned views work
    g.wrap_ct(lvl, [buf[0][4:], buf[1][4:]])
