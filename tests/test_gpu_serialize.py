"""Residue serialization (chd_ct_serialize / chd_evk_serialize): a
ciphertext (two or three parts, any level, with aux primes) and an
evaluation key (full basis and the dense-to-sparse basis) survive a round
trip bit for bit with their metadata; damaged buffers, buffers of another
ring degree and buffers over other primes are refused with an error."""
import json

import numpy as np
import pytest

import cheddar_b200 as chd
from gpu_common import mult_key, pair, param_json, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _same(a, b):
    assert a.info() == b.info()
    for x, y in zip(a.numpy(), b.numpy()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("level", [22, 7, 0])
def test_ciphertext_round_trip(cuda_ok, level):
    o, g = pair(KS)
    ct = g.import_ct(level, uniform_parts(KS, level, 50 + level), scale=2.0 ** 30 * 1.5, num_slots=1 << 12)
    _same(ct, g.load_ct(ct.serialize()))
    three = g.Mult(ct, ct)  # tensor: three parts
    assert three.info()["has_rx"]
    _same(three, g.load_ct(three.serialize()))


def test_key_round_trip(cuda_ok):
    o, g = pair(KS)
    _, k = mult_key(KS)
    data = k.serialize()
    back = g.load_evk(data)
    assert back.info() == k.info()
    for x, y in zip(k.numpy(), back.numpy()):
        assert np.array_equal(x, y)
    cl = chd.Client(g, 5)
    dts, _ = cl.sse_keys()
    back = g.load_evk(dts.serialize())
    assert back.info() == dts.info()


def test_bad_buffers_are_refused(cuda_ok):
    o, g = pair(KS)
    ct = g.import_ct(5, uniform_parts(KS, 5, 7))
    data = bytearray(ct.serialize())
    for bad, code in [(b"XXXXXXXX" + bytes(data[8:]), 8), (bytes(data[:-4]), 8), (bytes(data[:20]), 8)]:
        with pytest.raises(chd.CheddarError) as e:
            g.load_ct(bad)
        assert e.value.code == code
    flipped = bytearray(data)
    flipped[48] ^= 0x40  # a prime of the list
    with pytest.raises(chd.CheddarError) as e:
        g.load_ct(bytes(flipped))
    assert e.value.code == 3
    # a context over other primes (the reference's bootparam_30 primes)
    other = chd.Context(json.dumps(param_json("ntt_bootparam30_p24.json")))
    with pytest.raises(chd.CheddarError) as e:
        other.load_ct(bytes(data))
    assert e.value.code == 3
    small = chd.Context(json.dumps(param_json(KS, 13)))
    with pytest.raises(chd.CheddarError) as e:
        small.load_ct(bytes(data))
    assert e.value.code == 3
    _, k = mult_key(KS)
    with pytest.raises(chd.CheddarError):
        g.load_ct(k.serialize())
    with pytest.raises(chd.CheddarError):
        g.load_evk(bytes(data))
