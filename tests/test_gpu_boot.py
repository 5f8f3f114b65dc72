"""Bootstrapping building blocks against the oracle, bit-exact: the encoder
(Encoder::Encode / EncodeConstant, src/core/Encode.cpp) including padding,
auxiliary primes and scales beyond 2^64, and ModUpToMax
(BootContext::ModUpToMax, src/extension/BootContext.cpp:186-270) from level
-1 to the top level, including the property that the base limbs come back
unchanged."""
import numpy as np
import pytest
import torch

from gpu_common import pair, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("level,num_aux,log_scale,length", [
    (22, 0, 30, 1 << 15), (22, 8, 60, 1 << 15), (5, 0, 40, 7), (0, 3, 30, 1), (-1, 0, 80, 256), (13, 8, 90, 1000)])
def test_encode_bit_exact(cuda_ok, level, num_aux, log_scale, length):
    o, g = pair(KS)
    rng = np.random.default_rng(level + 100 * num_aux + length)
    msg = (rng.random(length) * 2 - 1) + 1j * (rng.random(length) * 2 - 1)
    ns = 1
    while ns < length:
        ns *= 2
    padded = np.zeros(ns, dtype=np.complex128)
    padded[:length] = msg
    ref = o.encode(level, 2.0 ** log_scale, padded, num_aux=num_aux)
    got = g.encode(level, 2.0 ** log_scale, msg, num_aux=num_aux)
    assert np.array_equal(_host(got), ref)


@pytest.mark.parametrize("value,log_scale", [(0.25, 30), (-0.0078125, 50), (-3.5, 62), (1e-9, 40), (123.456, 70),
                                             (0.0, 30)])
def test_encode_const_bit_exact(cuda_ok, value, log_scale):
    o, g = pair(KS)
    for level, num_aux in [(22, 0), (7, 8), (-1, 0)]:
        assert np.array_equal(g.encode_const(level, 2.0 ** log_scale, value, num_aux),
                              o.encode_const(level, 2.0 ** log_scale, value, num_aux))


# ModUpToMax without sparse-secret encapsulation needs a parameter set whose
# dense and sparse Hamming weights agree (the key-switching set has 192 > 32)
PLAIN = "boot_l34_a12.json"


def test_modup_to_max_bit_exact(cuda_ok):
    o, g = pair(PLAIN, 12)
    bx, ax = uniform_parts(PLAIN, -1, 4242, log_n=12)
    ref_b, ref_a = o.modup_to_max(bx, ax)
    r = g.ModUpToMax(g.import_ct(-1, [bx, ax]))
    parts = r.numpy()
    assert np.array_equal(parts[0], ref_b) and np.array_equal(parts[1], ref_a)
    # in place, twice in a row
    c = g.import_ct(-1, [bx, ax])
    g.ModUpToMax(c, res=c)
    parts = c.numpy()
    assert np.array_equal(parts[0], ref_b) and np.array_equal(parts[1], ref_a)


def test_modup_to_max_keeps_base_limbs(cuda_ok):
    # the lift is congruent to the input modulo the base primes, which are the
    # first primes of the top level: those limbs come back unchanged
    o, g = pair(PLAIN, 12)
    bx, ax = uniform_parts(PLAIN, -1, 777, log_n=12)
    r = g.ModUpToMax(g.import_ct(-1, [bx, ax])).numpy()
    nb = o.num_q(-1)
    assert np.array_equal(r[0][:nb], bx) and np.array_equal(r[1][:nb], ax)
