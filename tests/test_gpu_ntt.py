"""GPU NTT / INTT against the oracle, bit-exact (config: N = 2^16, the 24
q primes + 8 aux primes of the key-switching parameter set; plus the
single-kernel path for N = 2^12 .. 2^15)."""
import numpy as np
import pytest
import torch

from gpu_common import pair

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("mont", [False, True])
def test_ntt_forward_all_primes(cuda_ok, mont):
    o, g = pair("keyswitch_l24_a8.json")
    lvl = o.max_level
    m, t = o.level_np(lvl)
    x = o.uniform(11, lvl, num_aux=o.alpha)
    d = _dev(x)
    g.ntt_raw(m, t, o.alpha, d, mont=mont)
    g.synchronize()
    assert np.array_equal(_host(d), o.ntt(lvl, x, num_aux=o.alpha, mont=mont))


@pytest.mark.parametrize("mont", [True, False])
def test_ntt_inverse_all_primes(cuda_ok, mont):
    o, g = pair("keyswitch_l24_a8.json")
    lvl = o.max_level
    m, t = o.level_np(lvl)
    x = o.uniform(12, lvl, num_aux=o.alpha)
    d = _dev(x)
    g.intt_raw(m, t, o.alpha, d, mont=mont)
    g.synchronize()
    assert np.array_equal(_host(d), o.intt(lvl, x, num_aux=o.alpha, mont=mont))


def test_ntt_roundtrip_batch(cuda_ok):
    """count > 1 consecutive polynomials, more rows than one launch holds"""
    o, g = pair("keyswitch_l24_a8.json")
    lvl = o.max_level
    m, t = o.level_np(lvl)
    xs = np.stack([o.uniform(20 + i, lvl, num_aux=o.alpha) for i in range(5)])
    d = _dev(xs)
    g.ntt_raw(m, t, o.alpha, d, mont=True, count=5)
    g.intt_raw(m, t, o.alpha, d, mont=True, count=5)
    g.synchronize()
    assert np.array_equal(_host(d).reshape(xs.shape), xs)


@pytest.mark.parametrize("log_n", [12, 13, 14, 15])
def test_ntt_small_degrees(cuda_ok, log_n):
    o, g = pair("keyswitch_l8_a3.json", log_n)
    lvl = o.max_level
    m, t = o.level_np(lvl)
    x = o.uniform(13, lvl, num_aux=o.alpha)
    d = _dev(x)
    g.ntt_raw(m, t, o.alpha, d, mont=True)
    g.synchronize()
    assert np.array_equal(_host(d), o.ntt(lvl, x, num_aux=o.alpha, mont=True))
    g.intt_raw(m, t, o.alpha, d, mont=False)
    g.synchronize()
    y = o.ntt(lvl, x, num_aux=o.alpha, mont=True)
    assert np.array_equal(_host(d), o.intt(lvl, y, num_aux=o.alpha, mont=False))


def test_ntt_edge_values(cuda_ok):
    """0, 1, q-1 and alternating extremes in every limb"""
    o, g = pair("keyswitch_l24_a8.json")
    lvl = o.max_level
    m, t = o.level_np(lvl)
    primes = o.primes(lvl, num_aux=o.alpha).astype(np.uint64)
    x = np.zeros((len(primes), o.n), dtype=np.uint64)
    x[:, 1::3] = 1
    x[:, 2::3] = (primes - 1)[:, None]
    x = x.astype(np.uint32)
    d = _dev(x)
    g.ntt_raw(m, t, o.alpha, d, mont=False)
    g.synchronize()
    assert np.array_equal(_host(d), o.ntt(lvl, x, num_aux=o.alpha, mont=False))
