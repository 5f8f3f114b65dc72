"""Full-slot bootstrapping (BootContext::Boot, src/extension/BootContext.cpp:
scale-up, ModUpToMax, CoeffToSlot, EvalMod on the real and imaginary parts,
SlotToCoeff) on the bootstrapping parameter set at N = 2^12 (2048 slots):
the GPU result equals the oracle running the same compiled program on its
own primitives, bit for bit, and decrypts to the input message (slots
uniform in [-1, 1] x [-1, 1]; precision reported in bits)."""
import functools

import numpy as np
import pytest

import cheddar_b200 as chd
from boot_oracle import Ct, run_program
from gpu_common import pair

pytestmark = pytest.mark.gpu
BOOT = "boot_l34_a12.json"
LOGN = 12


@functools.lru_cache(maxsize=None)
def _setup():
    o, g = pair(BOOT, LOGN)
    bc = chd.BootContext(g)
    s = o.gen_secret(99, 32)
    mk = o.gen_mult_key(77, s)
    ck = o.gen_conj_key(78, s)
    rks = {r: o.gen_rot_key(1000 + r, s, r) for r in sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True)))}
    keys = chd.EvkMap(g)
    keys.set_mult(g.evk(*mk))
    keys.set_conjugation(g.evk(*ck))
    for r, k in rks.items():
        keys.set_rotation(r, g.evk(*k))
    return o, g, bc, s, mk, ck, rks, keys


def test_boot_levels(cuda_ok):
    o, g, bc, *_ = _setup()
    assert bc.cts_start == o.max_level == 34
    assert (bc.eval_mod_start, bc.stc_start, bc.end_level) == (30, 22, 19)
    assert bc.log_scaleup >= 0


def test_boot_bit_exact_and_precision(cuda_ok):
    o, g, bc, s, mk, ck, rks, keys = _setup()
    rng = np.random.default_rng(2024)
    half = o.n // 2
    msg = (rng.random(half) * 2 - 1) + 1j * (rng.random(half) * 2 - 1)
    sc0 = o.scale(0)
    bx, ax = o.encrypt(5, s, 0, o.encode(0, sc0, msg))
    res = bc.Boot(g.import_ct(0, [bx, ax], sc0), keys)
    parts = res.numpy()
    ref = run_program(o, bc.json(), Ct(0, [bx, ax], sc0), mult_key=mk, conj_key=ck, rot_keys=rks,
                      lts=bc.transforms())
    assert ref.level == bc.end_level
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
    info = res.info()
    assert abs(info["scale"] - bc.final_scale) <= 1e-9 * bc.final_scale
    dec = o.decode(bc.end_level, bc.final_scale, o.decrypt(s, bc.end_level, parts), half)
    err = np.abs(dec - msg).max()
    bits = -np.log2(err)
    print(f"bootstrapping precision: {bits:.2f} bits (max error {err:.3e})")
    assert bits > 10, bits


def test_boot_min_ks_bit_exact_and_precision(cuda_ok):
    # Boot(res, input, evk_map, min_ks = true): the reference's Boot-MinKS
    # test (unittest/Bootstrapping.cpp:34-36); two keys per transform
    o, g, bc, s, mk, ck, rks, keys = _setup()
    assert len(bc.rotations(min_ks=True)) < len(bc.rotations())
    rng = np.random.default_rng(4048)
    half = o.n // 2
    msg = (rng.random(half) * 2 - 1) + 1j * (rng.random(half) * 2 - 1)
    sc0 = o.scale(0)
    bx, ax = o.encrypt(8, s, 0, o.encode(0, sc0, msg))
    res = bc.Boot(g.import_ct(0, [bx, ax], sc0), keys, min_ks=True)
    parts = res.numpy()
    ref = run_program(o, bc.json(), Ct(0, [bx, ax], sc0), mult_key=mk, conj_key=ck, rot_keys=rks,
                      lts=bc.transforms(), min_ks=True)
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
    dec = o.decode(bc.end_level, bc.final_scale, o.decrypt(s, bc.end_level, parts), half)
    err = np.abs(dec - msg).max()
    print(f"min-KS bootstrapping precision: {-np.log2(err):.2f} bits")
    assert -np.log2(err) > 10


def test_boot_batch_equals_single(cuda_ok):
    # BootBatch: every key switch, rescale and linear transform of the
    # program runs once over the batch; each result equals a single Boot,
    # also with the min-KS transforms and with a result aliasing its input
    o, g, bc, s, mk, ck, rks, keys = _setup()
    rng = np.random.default_rng(77)
    half = o.n // 2
    sc0 = o.scale(0)
    cts = []
    for i in range(3):
        msg = (rng.random(half) * 2 - 1) + 1j * (rng.random(half) * 2 - 1)
        bx, ax = o.encrypt(40 + i, s, 0, o.encode(0, sc0, msg))
        cts.append((bx, ax))
    for min_ks in (False, True):
        single = [bc.Boot(g.import_ct(0, list(c), sc0), keys, min_ks=min_ks).numpy() for c in cts]
        ins = [g.import_ct(0, list(c), sc0) for c in cts]
        outs = bc.BootBatch(ins, keys, min_ks=min_ks)
        for a, b in zip(outs, single):
            p = a.numpy()
            assert np.array_equal(p[0], b[0]) and np.array_equal(p[1], b[1])
        # in place: results alias the inputs
        ins = [g.import_ct(0, list(c), sc0) for c in cts]
        bc.BootBatch(ins, keys, res_list=ins, min_ks=min_ks)
        for a, b in zip(ins, single):
            p = a.numpy()
            assert np.array_equal(p[0], b[0]) and np.array_equal(p[1], b[1])
