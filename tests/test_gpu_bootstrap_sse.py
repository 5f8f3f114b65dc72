"""Bootstrapping with sparse-secret encapsulation (the reference's
bootparam_*.json setting: dense Hamming weight above the sparse one).
ModUpToMax runs the dense-to-sparse key switch at level -1, the exact lift
and the single-digit sparse-to-dense key switch (BootContext.cpp:186-270);
the GPU result equals the oracle's restatement bit for bit, a full-slot
bootstrap at N = 2^12 equals the oracle running the same program and
decrypts to its input, and an input above level 0 is first brought down
with LevelDown (Context.cpp:917-929).  Two parameter shapes: the 30-bit one
(48 q primes, no terminal primes) and the reference's 40-bit one (4
terminal + 43 main primes, rational rescale)."""
import functools

import numpy as np
import pytest

import cheddar_b200 as chd
from boot_oracle import Ct, gen_sse_keys, run_program
from gpu_common import pair, uniform_parts

pytestmark = pytest.mark.gpu
BOOTS = ["boot_l34_a12_sse.json", "boot40_l28_a12.json"]
LOGN = 12


@functools.lru_cache(maxsize=None)
def _setup(name):
    o, g = pair(name, LOGN)
    bc = chd.BootContext(g)
    dense = o.gen_secret(199, o.n // 2)
    sparse = o.gen_secret(299, 32)
    mk = o.gen_mult_key(177, dense)
    ck = o.gen_conj_key(178, dense)
    rks = {r: o.gen_rot_key(2000 + r, dense, r) for r in bc.rotations()}
    dts, std = gen_sse_keys(o, 377, dense, sparse)
    m, t = o.level_np(-1)
    keys = chd.EvkMap(g)
    keys.set_mult(g.evk(*mk))
    keys.set_conjugation(g.evk(*ck))
    for r, k in rks.items():
        keys.set_rotation(r, g.evk(*k))
    keys.set_dense_to_sparse(chd.EvaluationKey(g, dts[0], dts[1], basis=(m, t, m + t)))
    keys.set_sparse_to_dense(chd.EvaluationKey(g, std[0], std[1], basis=(o.L - o.max_ter, o.max_ter, o.alpha)))
    return o, g, bc, dense, mk, ck, rks, (dts, std), keys


@pytest.mark.parametrize("name", BOOTS)
def test_modup_to_max_sse_bit_exact(cuda_ok, name):
    o, g, bc, dense, mk, ck, rks, sse, keys = _setup(name)
    bx, ax = uniform_parts(name, -1, 31, log_n=LOGN)
    ref_b, ref_a = o.modup_to_max_sse(bx, ax, sse[0], sse[1])
    r = g.ModUpToMax(g.import_ct(-1, [bx, ax]), keys=keys).numpy()
    assert np.array_equal(r[0], ref_b) and np.array_equal(r[1], ref_a)


@pytest.mark.parametrize("name", BOOTS)
@pytest.mark.parametrize("in_level", [0, 3])
def test_boot_sse_bit_exact_and_precision(cuda_ok, name, in_level):
    o, g, bc, dense, mk, ck, rks, sse, keys = _setup(name)
    rng = np.random.default_rng(2025 + in_level)
    half = o.n // 2
    msg = (rng.random(half) * 2 - 1) + 1j * (rng.random(half) * 2 - 1)
    sc = o.scale(in_level)
    bx, ax = o.encrypt(9, dense, in_level, o.encode(in_level, sc, msg))
    res = bc.Boot(g.import_ct(in_level, [bx, ax], sc), keys)
    parts = res.numpy()
    dec = o.decode(bc.end_level, bc.final_scale, o.decrypt(dense, bc.end_level, parts), half)
    err = np.abs(dec - msg).max()
    print(f"{name}: bootstrapping with encapsulation from level {in_level}: {-np.log2(err):.2f} bits")
    assert -np.log2(err) > 10
    if in_level == 0:
        ref = run_program(o, bc.json(), Ct(0, [bx, ax], sc), mult_key=mk, conj_key=ck, rot_keys=rks,
                          lts=bc.transforms(), sse_keys=sse)
        assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
