"""The tensor-core engines of the fused ModUp / ModDown column pass (base
conversion as INT8 byte-limb MMAs on tcgen05, int32 accumulation in TMEM;
128-thread tiles, and 256-thread tiles for up to 12 sources) give the same
residues as the oracle and as the CUDA-core engine, bit for bit: raw ModUp / ModDown / Rescale, HMult with relinearisation and rescale,
batches, rotations, hoisted rotations, and a full-slot bootstrap at
N = 2^16 (every ModUp / ModDown / rescale of the bootstrapping program)."""
import contextlib
import json
import os

import numpy as np
import pytest
import torch

import cheddar_b200 as chd
from gpu_common import mult_key, pair, rot_key, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"
TC_ENGINES = [chd.BCONV_TENSOR_CORE, chd.BCONV_TENSOR_CORE_WIDE]
ALL_ENGINES = (chd.BCONV_CUDA_CORE, chd.BCONV_TENSOR_CORE, chd.BCONV_TENSOR_CORE_WIDE)


@contextlib.contextmanager
def engine(ctx, e):
    old = ctx.ks_engine
    ctx.ks_engine = e
    try:
        yield
    finally:
        ctx.ks_engine = old


def _eq(gpu_ct, ref_parts):
    parts = gpu_ct.numpy()
    for a, b in zip(parts, ref_parts):
        assert np.array_equal(a, b)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


def test_engine_setting(cuda_ok):
    o, g = pair(KS)
    assert g.ks_engine in (chd.BCONV_CUDA_CORE, chd.BCONV_TENSOR_CORE)
    with engine(g, chd.BCONV_TENSOR_CORE):
        assert g.ks_engine == chd.BCONV_TENSOR_CORE
        with pytest.raises(chd.CheddarError):
            g.ks_engine = 7
        assert g.ks_engine == chd.BCONV_TENSOR_CORE
    with engine(g, chd.BCONV_TENSOR_CORE_WIDE):
        assert g.ks_engine == chd.BCONV_TENSOR_CORE_WIDE


@pytest.mark.parametrize("eng", TC_ENGINES)
@pytest.mark.parametrize("level", [22, 21, 15, 6, 0])
def test_modup_moddown_tc(cuda_ok, level, eng):
    o, g = pair(KS)
    with engine(g, eng):
        x = o.uniform(30 + level, level)
        mu = torch.zeros((o.beta(level), o.num_q(level) + o.alpha, o.n), dtype=torch.int32, device="cuda")
        g.modup_raw(level, _dev(x), mu)
        g.synchronize()
        ref = o.modup(level, x)
        assert np.array_equal(_host(mu).reshape(ref.shape), ref)
        xa = np.stack([o.uniform(40 + level + i, level, num_aux=o.alpha) for i in range(2)])
        out = torch.zeros((2, o.num_q(level), o.n), dtype=torch.int32, device="cuda")
        g.moddown_raw(level, chd.CHD_MODDOWN, _dev(xa), out, npoly=2)
        g.synchronize()
        for i in range(2):
            assert np.array_equal(_host(out[i]), o.moddown(level, xa[i]))
        if level > 0:
            out1 = torch.zeros((o.num_q(level - 1), o.n), dtype=torch.int32, device="cuda")
            g.moddown_raw(level, chd.CHD_RESCALE, _dev(x), out1)
            g.synchronize()
            assert np.array_equal(_host(out1), o.rescale(level, x))
            g.moddown_raw(level, chd.CHD_MODDOWN_RESCALE, _dev(xa[0]), out1)
            g.synchronize()
            assert np.array_equal(_host(out1), o.moddown_rescale(level, xa[0]))


@pytest.mark.parametrize("eng", TC_ENGINES)
@pytest.mark.parametrize("level,rescale", [(22, True), (22, False), (13, True), (1, True)])
def test_hmult_tc(cuda_ok, level, rescale, eng):
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    a = uniform_parts(KS, level, 100 + level)
    b = uniform_parts(KS, level, 200 + level)
    with engine(g, eng):
        res = g.HMult(g.import_ct(level, a), g.import_ct(level, b), key, rescale=rescale)
        _eq(res, o.hmult(level, a, b, (kb, ka), rescale=rescale))


def test_hmult_batch_mixed_levels_tc(cuda_ok):
    # one launch per stage over ciphertexts at uneven levels, tensor-core
    # column passes; equal to the CUDA-core engine and to the oracle
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    levels = [20, 16, 9, 22, 5]
    pairs = [(uniform_parts(KS, l, 300 + i), uniform_parts(KS, l, 400 + i)) for i, l in enumerate(levels)]
    outs = {}
    for e in ALL_ENGINES:
        with engine(g, e):
            ga = [g.import_ct(l, a) for l, (a, _) in zip(levels, pairs)]
            gb = [g.import_ct(l, b) for l, (_, b) in zip(levels, pairs)]
            outs[e] = [r.numpy() for r in g.HMultBatch(ga, gb, key, rescale=True)]
    for i, (l, (a, b)) in enumerate(zip(levels, pairs)):
        ref = o.hmult(l, a, b, (kb, ka), rescale=True)
        for e in outs:
            for x, y in zip(outs[e][i], ref):
                assert np.array_equal(x, y)


@pytest.mark.parametrize("eng", TC_ENGINES)
@pytest.mark.parametrize("rot", [1, 1234, 32767])
def test_hrot_tc(cuda_ok, rot, eng):
    o, g = pair(KS)
    (kb, ka), key = rot_key(KS, rot)
    lvl = 21
    a = uniform_parts(KS, lvl, 700)
    with engine(g, eng):
        _eq(g.HRot(g.import_ct(lvl, a), key, rot), o.hrot(lvl, a, (kb, ka), rot))


@pytest.mark.parametrize("eng", TC_ENGINES)
def test_hoisted_rotations_tc(cuda_ok, eng):
    o, g = pair(KS)
    lvl = o.max_level
    offs = [1, 2, 3, 4, 16, 1024, 32767]
    a = uniform_parts(KS, lvl, 900)
    keys = [rot_key(KS, r) for r in offs]
    with engine(g, eng):
        ga = g.import_ct(lvl, a)
        outs = g.HoistedRotate(ga, [k[1] for k in keys], offs)
        hb, ha = o.hoisted_rotate(lvl, a, [k[0] for k in keys], offs)
        for i in range(len(offs)):
            _eq(outs[i], [hb[i], ha[i]])
        _eq(g.ModDown(outs[2]), o.hrot(lvl, a, keys[2][0], offs[2]))


def test_bootstrap_n16_engines_equal(cuda_ok):
    """Full-slot bootstrap at N = 2^16 on the bootstrapping parameter set
    (alpha = 12: 12-source column passes) with uniform random evaluation
    keys: the tensor-core engine's output equals the CUDA-core engine's."""
    params = json.load(open(os.path.join(chd.PARAM_DIR, "boot_l34_a12.json")))
    ctx = chd.Context(json.dumps(params))
    bc = chd.BootContext(ctx)
    n, L, a = ctx.n, ctx.L, ctx.alpha
    beta = -(-L // a)
    allp = torch.tensor(list(reversed(params.get("terminal_primes", []))) + params["main_primes"] +
                        params["auxiliary_primes"], dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(99)

    def uniform(rows):
        q = allp[torch.tensor(rows, device="cuda", dtype=torch.int64)][:, None]
        r = torch.randint(0, 2 ** 62, (len(rows), n), generator=gen, device="cuda", dtype=torch.int64)
        r = (r % q).to(torch.int32)
        torch.cuda.synchronize()  # the context works on its own stream
        return r

    kg = list(ctx.gidx(*ctx.level_np(ctx.max_level), a))
    keys = chd.EvkMap(ctx)
    held = []

    def ukey():
        kb = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        ka = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        torch.cuda.synchronize()
        k = chd.EvaluationKey(ctx, kb, ka, on_device=True)
        held.append(k)
        return k

    keys.set_mult(ukey())
    keys.set_conjugation(ukey())
    for r in bc.rotations():
        keys.set_rotation(r, ukey())
    g0 = list(ctx.gidx(*ctx.level_np(0), 0))
    ct = ctx.import_ct(0, [uniform(g0), uniform(g0)], on_device=True, scale=ctx.scale(0))
    torch.cuda.synchronize()
    res = {}
    for e in ALL_ENGINES:
        with engine(ctx, e):
            res[e] = bc.Boot(ct, keys).numpy()
    ctx.synchronize()
    for e in (chd.BCONV_TENSOR_CORE, chd.BCONV_TENSOR_CORE_WIDE):
        for x, y in zip(res[chd.BCONV_CUDA_CORE], res[e]):
            assert np.array_equal(x, y)


BOOT = "boot_l34_a12.json"


@pytest.mark.parametrize("eng", ["cuda", "tensor", "tensor_wide"])
@pytest.mark.parametrize("level", [34, 30, 22, 10])
def test_boot_params_column_passes(cuda_ok, eng, level):
    """Bootstrapping parameter set at N = 2^16 (alpha = 12): ModUp digits of
    12 primes, ModDown from 12 auxiliary primes, and the merged ModDown +
    Rescale with 13 sources (one prime dropped) or 14 (two primes dropped,
    levels above 24), whose last sources are held in registers; every
    engine equals the oracle."""
    o, g = pair(BOOT)
    e = {"cuda": chd.BCONV_CUDA_CORE, "tensor": chd.BCONV_TENSOR_CORE,
         "tensor_wide": chd.BCONV_TENSOR_CORE_WIDE}[eng]
    with engine(g, e):
        x = o.uniform(130 + level, level)
        mu = torch.zeros((o.beta(level), o.num_q(level) + o.alpha, o.n), dtype=torch.int32, device="cuda")
        g.modup_raw(level, _dev(x), mu)
        g.synchronize()
        ref = o.modup(level, x)
        assert np.array_equal(_host(mu).reshape(ref.shape), ref)
        xa = o.uniform(140 + level, level, num_aux=o.alpha)
        out = torch.zeros((o.num_q(level), o.n), dtype=torch.int32, device="cuda")
        g.moddown_raw(level, chd.CHD_MODDOWN, _dev(xa), out)
        g.synchronize()
        assert np.array_equal(_host(out), o.moddown(level, xa))
        out1 = torch.zeros((o.num_q(level - 1), o.n), dtype=torch.int32, device="cuda")
        g.moddown_raw(level, chd.CHD_MODDOWN_RESCALE, _dev(xa), out1)
        g.synchronize()
        assert np.array_equal(_host(out1), o.moddown_rescale(level, xa))
        g.moddown_raw(level, chd.CHD_RESCALE, _dev(x), out1)
        g.synchronize()
        assert np.array_equal(_host(out1), o.rescale(level, x))


def test_auto_engine(cuda_ok):
    """CHD_BCONV_AUTO: the first launch of each shape runs and times both
    engines, later ones use the faster; every result equals the oracle's
    (single HMult, a batch, raw ModUp / ModDown, a rotation)."""
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    with engine(g, chd.BCONV_AUTO):
        assert g.ks_engine == chd.BCONV_AUTO
        for rep in range(2):  # first call tunes, second uses the cache
            lvl = 22
            a = uniform_parts(KS, lvl, 1100 + rep)
            b = uniform_parts(KS, lvl, 1200 + rep)
            _eq(g.HMult(g.import_ct(lvl, a), g.import_ct(lvl, b), key, rescale=True),
                o.hmult(lvl, a, b, (kb, ka), rescale=True))
            pairs = [(uniform_parts(KS, 20, 1300 + 10 * rep + i), uniform_parts(KS, 20, 1400 + 10 * rep + i))
                     for i in range(4)]
            outs = g.HMultBatch([g.import_ct(20, x) for x, _ in pairs], [g.import_ct(20, y) for _, y in pairs], key,
                                rescale=True)
            for (x, y), r in zip(pairs, outs):
                _eq(r, o.hmult(20, x, y, (kb, ka), rescale=True))
            x = o.uniform(30 + rep, 15)
            mu = torch.zeros((o.beta(15), o.num_q(15) + o.alpha, o.n), dtype=torch.int32, device="cuda")
            g.modup_raw(15, _dev(x), mu)
            g.synchronize()
            ref = o.modup(15, x)
            assert np.array_equal(_host(mu).reshape(ref.shape), ref)
        (rb, ra), rk = rot_key(KS, 5)
        a = uniform_parts(KS, 21, 1500)
        _eq(g.HRot(g.import_ct(21, a), rk, 5), o.hrot(21, a, (rb, ra), 5))


def test_hmult_and_hrot_every_level_both_engines(cuda_ok):
    # every level of the key-switching set (1 .. 22, digit counts 1 .. 3,
    # ModDownAndRescale constants of each level) on both column-pass engines,
    # against the oracle: HMult with rescale, and a rotation
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    (rb, ra), rkey = rot_key(KS, 5)
    for lvl in range(1, o.max_level + 1):
        a = uniform_parts(KS, lvl, 900 + lvl)
        b = uniform_parts(KS, lvl, 950 + lvl)
        ref_m = o.hmult(lvl, a, b, (kb, ka), rescale=True)
        ref_r = o.hrot(lvl, a, (rb, ra), 5)
        for e in ALL_ENGINES:
            with engine(g, e):
                _eq(g.HMult(g.import_ct(lvl, a), g.import_ct(lvl, b), key, rescale=True), ref_m)
                _eq(g.HRot(g.import_ct(lvl, a), rkey, 5), ref_r)


def test_terminal_primes_n16_every_level_both_engines(cuda_ok):
    # the terminal-prime set (rational rescale, levels alternating between
    # 0, 2 and 4 terminal primes) at its own N = 2^16, where the key switches
    # take the fused pipeline: HMult with rescale and a rotation at every
    # level, both column-pass engines, against the oracle
    rat = "rational_t4_m10_a6.json"
    o, g = pair(rat)
    assert g.n == 65536
    (kb, ka), key = mult_key(rat)
    (rb, ra), rkey = rot_key(rat, 3)
    for lvl in range(1, o.max_level + 1):
        a = uniform_parts(rat, lvl, 1100 + lvl)
        b = uniform_parts(rat, lvl, 1150 + lvl)
        ref_m = o.hmult(lvl, a, b, (kb, ka), rescale=True)
        ref_r = o.hrot(lvl, a, (rb, ra), 3)
        for e in ALL_ENGINES:
            with engine(g, e):
                _eq(g.HMult(g.import_ct(lvl, a), g.import_ct(lvl, b), key, rescale=True), ref_m)
                _eq(g.HRot(g.import_ct(lvl, a), rkey, 3), ref_r)


def test_moddown_batch_equals_single(cuda_ok):
    """ModDownBatch of the 30 hoisted rotations of one ciphertext (one fused
    pipeline for all 60 polynomials) equals ModDown of each, and the oracle's
    HRot."""
    o, g = pair(KS)
    lvl = o.max_level
    half = o.n // 2
    offs = sorted({(s * (1 << k)) % half for k in range(15) for s in (1, -1)} | {1, 2, 3, 4})
    a = uniform_parts(KS, lvl, 950)
    keys = [rot_key(KS, r) for r in offs]
    ga = g.import_ct(lvl, a)
    qp = g.HoistedRotate(ga, [k[1] for k in keys], offs)
    batch = g.ModDownBatch(qp)
    for i in (0, 7, 29):
        _eq(batch[i], g.ModDown(qp[i]).numpy())
    _eq(batch[3], o.hrot(lvl, a, keys[3][0], offs[3]))
