"""CPU checks of the oracle: definitional known-answer tests, the
reference's accumulation schedule, and the reference's own decryption-error
criterion (|error| <= 1e-3 per slot, unittest/Testbed.h:93,294-365)."""
import os

import numpy as np
import pytest

import pyoracle as po

PARAMS = os.path.join(os.path.dirname(__file__), "..", "cheddar-fhe_b200", "params")


def _oracle(name, log_n=12):
    return po.Oracle(po.load_param_json(os.path.join(PARAMS, name)), log_degree=log_n)


def _brev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2)


def test_ntt_is_evaluation_at_odd_powers():
    o = _oracle("keyswitch_l8_a3.json")
    n, g = o.n, 2
    q = int(o.all_primes()[g])
    a = np.random.default_rng(1).integers(0, q, n, dtype=np.uint64).astype(np.uint32)
    A = o.ntt_limb(g, a, mont=False)
    psi = po.lib().orc_primitive_root(2 * n, q)
    for k in (0, 1, 2, 3, 100, n // 2, n - 1):
        w = pow(psi, 2 * _brev(k, o.log_n) + 1, q)
        v, x = 0, 1
        for i in range(n):
            v = (v + int(a[i]) * x) % q
            x = x * w % q
        assert v == int(A[k])


def test_ntt_negacyclic_convolution():
    o = _oracle("keyswitch_l8_a3.json")
    n, g = o.n, 5
    q = int(o.all_primes()[g])
    rng = np.random.default_rng(2)
    a = rng.integers(0, q, n, dtype=np.uint64)
    b = np.zeros(n, dtype=np.uint64)
    b[rng.integers(0, n, 8)] = rng.integers(0, q, 8, dtype=np.uint64)
    c = np.zeros(n, dtype=object)
    for j in np.nonzero(b)[0]:
        for i in range(n):
            k = i + j
            v = int(a[i]) * int(b[j])
            if k >= n:
                c[k - n] -= v
            else:
                c[k] += v
    c = np.array([int(x) % q for x in c], dtype=np.uint64).astype(np.uint32)
    A = o.ntt_limb(g, a.astype(np.uint32), mont=True)
    B = o.ntt_limb(g, b.astype(np.uint32), mont=False)
    L = po.lib()
    qi = L.orc_inv_mod_base(q)
    C_ = np.array([L.orc_mont_mult(int(x), int(y), q, qi) for x, y in zip(A, B)], dtype=np.uint32)
    assert np.array_equal(o.intt_limb(g, C_, mont=False), c)


def test_ntt_roundtrip_all_primes():
    o = _oracle("keyswitch_l24_a8.json")
    lvl = o.max_level
    x = o.uniform(7, lvl, num_aux=o.alpha)
    y = o.intt(lvl, o.ntt(lvl, x, num_aux=o.alpha, mont=True), num_aux=o.alpha, mont=True)
    assert np.array_equal(x, y)


@pytest.mark.parametrize("K", [1, 2, 3, 4, 5, 7, 8, 9, 12, 13, 16])
def test_bconv_reference_schedule_equivalence(K):
    """The reference's int64 schedule (renormalise every 4 terms, lazy
    Montgomery) gives the exact residue for centred inputs of main/aux-sized
    sources — the property the bit-exact GPU kernels rely on."""
    p = po.load_param_json(os.path.join(PARAMS, "keyswitch_l24_a8.json"))
    o = po.Oracle(p, log_degree=12)
    primes = o.all_primes()
    src, dst = primes[:K], primes[K:K + 8]
    if K >= 8:
        src = np.concatenate([primes[24:32], primes[: K - 8]])
        dst = primes[K - 8:K]
    T = o.bconv_table(src, dst)
    rng = np.random.default_rng(K)
    xt = np.stack([rng.integers(-(int(q) // 2), int(q) // 2 + 1, o.n) for q in src]).astype(np.int32)
    exact = o.bconv(xt, T, dst)
    sched = o.bconv(xt, T, dst, ref_schedule=True)
    assert np.array_equal(exact, sched)
    # definitional check on a few columns: sum_k xt_k * qhat_k * R mod p
    for m, pm in enumerate(dst):
        pm = int(pm)
        for j in (0, 17, o.n - 1):
            acc = 0
            for k, qk in enumerate(src):
                qhat = 1
                for jj, qj in enumerate(src):
                    if jj != k:
                        qhat = qhat * int(qj) % pm
                acc += int(xt[k, j]) * qhat
            assert (acc << 32) % pm == int(exact[m, j])


def _roundtrip_setup(name, log_n=12, h=64):
    o = _oracle(name, log_n)
    s = o.gen_secret(11, h)
    return o, s


def test_encrypt_decrypt_precision():
    o, s = _roundtrip_setup("keyswitch_l8_a3.json")
    rng = np.random.default_rng(3)
    lvl = o.max_level
    msg = rng.random(o.n // 2) + 1j * rng.random(o.n // 2)
    pt = o.encode(lvl, o.scale(lvl), msg)
    ct = o.encrypt(5, s, lvl, pt)
    out = o.decode(lvl, o.scale(lvl), o.decrypt(s, lvl, ct), o.n // 2)
    assert np.abs(out - msg).max() < 1e-3


@pytest.mark.parametrize("rescale", [True, False])
def test_hmult_decrypts(rescale):
    o, s = _roundtrip_setup("keyswitch_l8_a3.json")
    mk = o.gen_mult_key(9, s)
    rng = np.random.default_rng(4)
    lvl = o.max_level
    m1 = rng.random(o.n // 2) + 1j * rng.random(o.n // 2)
    m2 = rng.random(o.n // 2) + 1j * rng.random(o.n // 2)
    sc = o.scale(lvl)
    c1 = o.encrypt(1, s, lvl, o.encode(lvl, sc, m1))
    c2 = o.encrypt(2, s, lvl, o.encode(lvl, sc, m2))
    r = o.hmult(lvl, c1, c2, mk, rescale=rescale)
    lo = lvl - 1 if rescale else lvl
    out_sc = sc * sc / (o.rescale_prime_prod(lvl) if rescale else 1.0)
    out = o.decode(lo, out_sc, o.decrypt(s, lo, r), o.n // 2)
    assert np.abs(out - m1 * m2).max() < 1e-3


def test_rotation_conjugation_and_hoisting():
    o, s = _roundtrip_setup("keyswitch_l8_a3.json")
    rng = np.random.default_rng(5)
    lvl = o.max_level
    m = rng.random(o.n // 2) + 1j * rng.random(o.n // 2)
    sc = o.scale(lvl)
    ct = o.encrypt(1, s, lvl, o.encode(lvl, sc, m))
    rots = [1, 2, 7, o.n // 2 - 3]
    keys = [o.gen_rot_key(100 + r, s, r) for r in rots]
    for r, k in zip(rots, keys):
        out = o.decode(lvl, sc, o.decrypt(s, lvl, o.hrot(lvl, ct, k, r)), o.n // 2)
        assert np.abs(out - np.roll(m, -r)).max() < 1e-3
    hb, ha = o.hoisted_rotate(lvl, ct, keys, rots)
    for i, (r, k) in enumerate(zip(rots, keys)):
        rb, ra = o.hrot(lvl, ct, k, r)
        assert np.array_equal(o.moddown(lvl, hb[i]), rb)
        assert np.array_equal(o.moddown(lvl, ha[i]), ra)
    ck = o.gen_conj_key(3, s)
    out = o.decode(lvl, sc, o.decrypt(s, lvl, o.hconj(lvl, ct, ck)), o.n // 2)
    assert np.abs(out - np.conj(m)).max() < 1e-3


def test_rational_rescale_chain():
    """Terminal primes with rational rescale: HMult + merged ModDown/Rescale
    down a level chain that alternately drops main and terminal primes."""
    o, s = _roundtrip_setup("rational_t4_m10_a6.json")
    mk = o.gen_mult_key(9, s)
    lvl = 7
    rng = np.random.default_rng(6)
    m = rng.random(o.n // 2) - 0.5
    # use a large scale so every rescale keeps enough precision
    sc = 2.0 ** 56
    ct = o.encrypt(1, s, lvl, o.encode(lvl, sc, m))
    one = o.encrypt(2, s, lvl, o.encode(lvl, 2.0 ** 56, np.ones(o.n // 2)))
    r = o.hmult(lvl, ct, one, mk, rescale=True)
    out_sc = sc * 2.0 ** 56 / o.rescale_prime_prod(lvl)
    out = o.decode(lvl - 1, out_sc, o.decrypt(s, lvl - 1, r), o.n // 2)
    assert np.abs(out - m).max() < 1e-3
