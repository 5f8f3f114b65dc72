"""The device encoder / decoder and the test-only client (the reference's
Encoder and UserInterface, src/core/Encode.cpp, src/UserInterface.cu):

* the device encoder equals the oracle's encoder residue for residue, and
  decoding an encoding returns the message (the decoder's doubles are pinned
  to the reference's own decoder in tests/test_gpu_refpin.py, case decode);
* the client's keys have the reference's structure: for every digit i of a
  key with encryption secret s' and target t,
  b_i + a_i s' - [digit rows] P t is one small error polynomial (the same
  integer coefficients, |e| <= 19, on every prime of the key basis) —
  checked on the CPU from the exported secret and key;
* keys and encryptions are reproducible from the seed and differ between
  seeds;
* encryption -> HMult / HRot / HConj with the client's keys -> decryption
  -> decoding gives the expected slots, and a full-slot bootstrap on the
  reference's bootparam_40.json with client keys (sparse-secret
  encapsulation included) decodes to its input at the reference's precision.
"""
import functools
import json
import os

import numpy as np
import pytest
import torch

import cheddar_b200 as chd
from boot_oracle import mont_mul
from gpu_common import pair, param_json

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _msg(seed, n, lo=0.0, hi=1.0):
    rng = np.random.default_rng(seed)
    return (rng.random(n) * (hi - lo) + lo) + 1j * (rng.random(n) * (hi - lo) + lo)


@pytest.mark.parametrize("level,ns", [(22, 1 << 15), (9, 1 << 12), (0, 256)])
def test_device_encoder_matches_oracle_and_decodes(cuda_ok, level, ns):
    o, g = pair(KS)
    msg = _msg(level, ns, -1, 1)
    sc = o.scale(level)
    pt = g.encode(level, sc, msg)
    g.synchronize()
    host = pt.cpu().numpy().view(np.uint32)
    assert np.array_equal(host, o.encode(level, sc, msg))
    dec = g.decode(level, sc, pt, ns)
    assert np.abs(dec - msg).max() < 1e-4
    assert np.abs(dec - o.decode(level, sc, host, ns)).max() < 1e-9


def _error_poly(o, rows_gidx, diff):
    """INTT of each row of `diff` (NTT Montgomery domain) as centred integers."""
    out = []
    for r, gi in enumerate(rows_gidx):
        q = int(o.all_primes()[gi])
        x = o.intt_limb(gi, diff[r], mont=True).astype(np.int64)
        out.append(np.where(x > q // 2, x - q, x))
    return np.stack(out)


def _check_key(o, key, s_enc, target, rows_gidx):
    """b_i + a_i s' - (digit rows) P t = the same small integers on every row."""
    kb, ka = key
    beta, rows = kb.shape[0], kb.shape[1]
    primes = o.all_primes()
    nq = rows - o.alpha
    aux_g = rows_gidx[nq:]
    for i in range(beta):
        diff = np.zeros((rows, o.n), dtype=np.uint32)
        for r, gi in enumerate(rows_gidx):
            q = int(primes[gi])
            v = (kb[i, r].astype(np.int64) + mont_mul(ka[i, r], s_enc[gi], q)) % q
            if i * o.alpha <= r < min((i + 1) * o.alpha, nq):
                p = 1
                for a in aux_g:
                    p = p * int(primes[a]) % q
                pm = (p << 32) % q
                v = (v - mont_mul(target[gi], np.full(o.n, pm, dtype=np.uint32), q)) % q
            diff[r] = v.astype(np.uint32)
        e = _error_poly(o, rows_gidx, diff)
        assert np.abs(e).max() <= 19
        assert (e == e[0]).all(), f"digit {i}: rows hold different error polynomials"
        assert np.abs(e[0]).max() >= 1  # not a zero error


@functools.lru_cache(maxsize=None)
def _small():
    o, g = pair("keyswitch_l8_a3.json", 12)
    return o, g, chd.Client(g, 1234)


def test_client_key_structure(cuda_ok):
    o, g, cl = _small()
    s = cl.secret()
    rows = list(range(o.nprimes))
    # secret: ternary with the dense Hamming weight, on every prime
    coeffs = _error_poly(o, rows, s)
    assert set(np.unique(coeffs[0])) <= {-1, 0, 1}
    assert (coeffs == coeffs[0]).all()
    assert int(np.count_nonzero(coeffs[0])) == g_dense(o)
    mk = cl.mult_key().numpy()
    s2 = np.stack([mont_mul(s[r], s[r], int(o.all_primes()[r])) for r in rows])
    _check_key(o, mk, s, s2, rows)
    for r in (1, 5, o.n // 2 - 1):
        rk = cl.rotation_key(r).numpy()
        sr = o.permute(o.max_level, o.n // 2 - r, s, num_aux=o.alpha)
        _check_key(o, rk, sr, s, rows)
    ck = cl.conjugation_key().numpy()
    sc = o.permute(o.max_level, -1, s, num_aux=o.alpha)
    _check_key(o, ck, sc, s, rows)


def g_dense(o):
    return o.params.get("dense_hamming_weight") or o.n // 2


def test_client_reproducible(cuda_ok):
    o, g, cl = _small()
    again = chd.Client(g, 1234)
    other = chd.Client(g, 1235)
    assert np.array_equal(cl.secret(), again.secret())
    assert not np.array_equal(cl.secret(), other.secret())
    a, b = cl.rotation_key(3).numpy(), again.rotation_key(3).numpy()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[1], other.rotation_key(3).numpy()[1])
    lvl = o.max_level
    pt = g.encode(lvl, o.scale(lvl), _msg(1, o.n // 2))
    c1, c2 = cl.encrypt(pt, lvl, o.scale(lvl), nonce=7), again.encrypt(pt, lvl, o.scale(lvl), nonce=7)
    assert all(np.array_equal(x, y) for x, y in zip(c1.numpy(), c2.numpy()))
    c3 = cl.encrypt(pt, lvl, o.scale(lvl), nonce=8)
    assert not np.array_equal(c1.numpy()[1], c3.numpy()[1])


def test_client_evaluate_decrypt(cuda_ok):
    o, g = pair(KS)
    cl = chd.Client(g, 99)
    mk, ck = cl.mult_key(), cl.conjugation_key()
    lvl = o.max_level
    half = o.n // 2
    m1, m2 = _msg(1, half), _msg(2, half)
    sc = o.scale(lvl)
    a = cl.encrypt(g.encode(lvl, sc, m1), lvl, sc, nonce=1)
    b = cl.encrypt(g.encode(lvl, sc, m2), lvl, sc, nonce=2)
    assert np.abs(cl.decrypt_decode(a) - m1).max() < 1e-5
    prod = cl.decrypt_decode(g.HMult(a, b, mk))
    assert np.abs(prod - m1 * m2).max() < 1e-3
    for r in (1, 7, half - 3):
        rot = cl.decrypt_decode(g.HRot(a, cl.rotation_key(r), r))
        assert np.abs(rot - np.roll(m1, -r)).max() < 1e-4
    conj = cl.decrypt_decode(g.HConj(a, ck))
    assert np.abs(conj - np.conj(m1)).max() < 1e-4


def test_client_bootstrap_bootparam40(cuda_ok):
    p = json.load(open(os.path.join(chd.PARAM_DIR, "bootparam_40.json")))
    g = chd.Context(json.dumps(p))
    bc = chd.BootContext(g)
    cl = chd.Client(g, 2024)
    keys = chd.EvkMap(g)
    keys.set_mult(cl.mult_key())
    keys.set_conjugation(cl.conjugation_key())
    for r in sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True))):
        keys.set_rotation(r, cl.rotation_key(r))
    dts, std = cl.sse_keys()
    keys.set_dense_to_sparse(dts)
    keys.set_sparse_to_dense(std)
    half = g.n // 2
    msg = _msg(5, half, -1, 1)
    sc0 = g.scale(0)
    ct = cl.encrypt(g.encode(0, sc0, msg), 0, sc0, nonce=3)
    for min_ks in (False, True):
        res = bc.Boot(ct, keys, min_ks=min_ks)
        dec = cl.decrypt_decode(res)
        err = float(np.abs(dec - msg).max())
        bits = -np.log2(err)
        assert bits >= 18.5, (min_ks, bits)
        import conftest
        conftest.REPORT.append(json.dumps({"client_keys_boot": "bootparam_40.json", "min_ks": min_ks,
                                           "precision_bits": round(float(bits), 2)}))
