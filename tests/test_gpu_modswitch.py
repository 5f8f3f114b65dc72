"""GPU base conversion and ModUp / ModDown / Rescale / ModDownAndRescale
against the oracle, bit-exact.  Covers the key-switching set at N = 2^16
(ragged last digit at lower levels) and the terminal-prime set with rational
rescale (restore / padding constants) at N = 2^12."""
import numpy as np
import pytest
import torch

import cheddar_b200 as chd
from gpu_common import pair

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    # the library works on its own stream: wait for it before torch reads
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("K,M", [(1, 24), (4, 12), (8, 24), (9, 23), (12, 4), (13, 19), (16, 16)])
def test_bconv_raw(cuda_ok, K, M):
    o, g = pair("keyswitch_l24_a8.json")
    primes = o.all_primes()
    rng = np.random.default_rng(K * 100 + M)
    gidx = rng.permutation(len(primes))
    src, dst = gidx[:K], gidx[K:K + M] if K + M <= len(primes) else gidx[-M:]
    xt = np.stack([rng.integers(-(int(primes[s]) // 2), int(primes[s]) // 2 + 1, o.n) for s in src]).astype(np.int32)
    out = torch.zeros((M, o.n), dtype=torch.int32, device="cuda")
    g.bconv_raw(torch.from_numpy(xt).cuda(), src, dst, out)
    g.synchronize()
    T = o.bconv_table(primes[src], primes[dst])
    assert np.array_equal(_host(out), o.bconv(xt, T, primes[dst]))


KS_LEVELS = [22, 21, 15, 6, 0]


@pytest.mark.parametrize("level", KS_LEVELS)
def test_modup(cuda_ok, level):
    o, g = pair("keyswitch_l24_a8.json")
    x = o.uniform(30 + level, level)
    beta = o.beta(level)
    out = torch.zeros((beta, o.num_q(level) + o.alpha, o.n), dtype=torch.int32, device="cuda")
    g.modup_raw(level, _dev(x), out)
    g.synchronize()
    ref = o.modup(level, x)
    assert np.array_equal(_host(out).reshape(ref.shape), ref)


@pytest.mark.parametrize("level", KS_LEVELS)
def test_moddown(cuda_ok, level):
    o, g = pair("keyswitch_l24_a8.json")
    x = np.stack([o.uniform(40 + level + i, level, num_aux=o.alpha) for i in range(2)])
    out = torch.zeros((2, o.num_q(level), o.n), dtype=torch.int32, device="cuda")
    g.moddown_raw(level, chd.CHD_MODDOWN, _dev(x), out, npoly=2)
    g.synchronize()
    for i in range(2):
        assert np.array_equal(_host(out[i]), o.moddown(level, x[i]))


@pytest.mark.parametrize("level", [22, 12, 1])
def test_rescale_and_merged(cuda_ok, level):
    o, g = pair("keyswitch_l24_a8.json")
    x = o.uniform(50 + level, level)
    out = torch.zeros((o.num_q(level - 1), o.n), dtype=torch.int32, device="cuda")
    g.moddown_raw(level, chd.CHD_RESCALE, _dev(x), out)
    g.synchronize()
    assert np.array_equal(_host(out), o.rescale(level, x))
    xa = o.uniform(60 + level, level, num_aux=o.alpha)
    g.moddown_raw(level, chd.CHD_MODDOWN_RESCALE, _dev(xa), out)
    g.synchronize()
    assert np.array_equal(_host(out), o.moddown_rescale(level, xa))


RATIONAL_LEVELS = list(range(1, 10))


@pytest.mark.parametrize("level", RATIONAL_LEVELS)
def test_rational_rescale_all_levels(cuda_ok, level):
    o, g = pair("rational_t4_m10_a6.json", 12)
    x = o.uniform(70 + level, level)
    out = torch.zeros((o.num_q(level - 1), o.n), dtype=torch.int32, device="cuda")
    g.moddown_raw(level, chd.CHD_RESCALE, _dev(x), out)
    g.synchronize()
    assert np.array_equal(_host(out), o.rescale(level, x))
    xa = o.uniform(80 + level, level, num_aux=o.alpha)
    g.moddown_raw(level, chd.CHD_MODDOWN_RESCALE, _dev(xa), out)
    g.synchronize()
    assert np.array_equal(_host(out), o.moddown_rescale(level, xa))
    out2 = torch.zeros((o.num_q(level), o.n), dtype=torch.int32, device="cuda")
    g.moddown_raw(level, chd.CHD_MODDOWN, _dev(xa), out2)
    g.synchronize()
    assert np.array_equal(_host(out2), o.moddown(level, xa))
    mu = torch.zeros((o.beta(level), o.num_q(level) + o.alpha, o.n), dtype=torch.int32, device="cuda")
    g.modup_raw(level, _dev(x), mu)
    g.synchronize()
    ref = o.modup(level, x)
    assert np.array_equal(_host(mu).reshape(ref.shape), ref)
