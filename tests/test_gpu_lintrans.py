"""Linear transforms with double hoisting (LinearTransform + HoistHandler,
src/extension/LinearTransform.cpp, src/extension/Hoist.cu) against the
oracle's restatement, bit-exact, on the three evaluation shapes: a single
giant step (swapped to baby steps only), the general baby-step / giant-step
path with giant step 0, and one without giant step 0.  The decrypted result
also matches the plaintext matrix-vector product (the reference's 1e-3
criterion, unittest/Testbed.h:93)."""
import numpy as np
import pytest

import cheddar_b200 as chd
from boot_oracle import lt_evaluate
from gpu_common import fresh_ct, pair, rot_key, secret

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"
LEVEL = 20


def _diags(idx, width, seed):
    rng = np.random.default_rng(seed)
    return {i: 0.3 * ((rng.random(width) * 2 - 1) + 1j * (rng.random(width) * 2 - 1)) for i in idx}


def _matvec(diags, v):
    w = len(v)
    out = np.zeros(w, dtype=np.complex128)
    for i, d in diags.items():
        out += d * np.roll(v, -i)
    return out


@pytest.mark.parametrize("idx,bs,gs", [([0, 1, 2], 3, 1), (list(range(16)), 4, 4), (list(range(8, 16)), 4, 4)])
def test_lintrans_bit_exact(cuda_ok, idx, bs, gs):
    o, g = pair(KS)
    width = o.n // 2
    diags = _diags(idx, width, seed=len(idx) * 7 + bs)
    pt_scale = o.rescale_prime_prod(LEVEL)
    lt = chd.LinearTransform(g, diags, LEVEL, pt_scale, bs, gs)
    rots = lt.rotations()
    keys = chd.EvkMap(g)
    host_keys = {}
    for r in rots:
        (kb, ka), k = rot_key(KS, r)
        keys.set_rotation(r, k)
        host_keys[r] = (kb, ka)
    (bx, ax), sc, msg = fresh_ct(KS, LEVEL, 31 + len(idx))
    res = lt.evaluate(g.import_ct(LEVEL, [bx, ax], sc), keys)
    (rb, ra), rscale = lt_evaluate(o, LEVEL, (bx, ax), sc, lt.plaintexts(), pt_scale, host_keys)
    parts = res.numpy()
    assert np.array_equal(parts[0], rb) and np.array_equal(parts[1], ra)
    info = res.info()
    assert abs(info["scale"] - rscale) <= 1e-9 * rscale
    dec = o.decode(LEVEL - 1, rscale, o.decrypt(secret(KS), LEVEL - 1, parts), width)
    assert np.abs(dec - _matvec(diags, msg)).max() < 1e-3


def test_lintrans_min_ks_bit_exact(cuda_ok):
    # the min-KS evaluation (two rotation keys: the baby and giant strides)
    o, g = pair(KS)
    width = o.n // 2
    diags = _diags(list(range(16)), width, seed=99)
    pt_scale = o.rescale_prime_prod(LEVEL)
    lt = chd.LinearTransform(g, diags, LEVEL, pt_scale, 4, 4)
    rots = lt.rotations(min_ks=True)
    assert rots == [1, 4]
    keys = chd.EvkMap(g)
    host_keys = {}
    for r in rots:
        (kb, ka), k = rot_key(KS, r)
        keys.set_rotation(r, k)
        host_keys[r] = (kb, ka)
    (bx, ax), sc, msg = fresh_ct(KS, LEVEL, 41)
    res = lt.evaluate(g.import_ct(LEVEL, [bx, ax], sc), keys, min_ks=True)
    (rb, ra), rscale = lt_evaluate(o, LEVEL, (bx, ax), sc, lt.plaintexts(), pt_scale, host_keys, min_ks=True)
    parts = res.numpy()
    assert np.array_equal(parts[0], rb) and np.array_equal(parts[1], ra)
    dec = o.decode(LEVEL - 1, rscale, o.decrypt(secret(KS), LEVEL - 1, parts), width)
    assert np.abs(dec - _matvec(diags, msg)).max() < 1e-3
