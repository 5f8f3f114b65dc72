"""Sparse-slot bootstrapping and the BootVariants (BootContext::Boot with
fewer than N/2 slots, src/extension/BootContext.cpp:321-362: Trace after
ModUpToMax, the extended 2n x 2n CoeffToSlot / SlotToCoeff phases of
EvalSpecialFFT.cpp:212-226, 268-282, one EvalMod on HConj(x) + x, the final
HRotAdd by n; kImaginaryRemoving's halved StC constant and closing
HConj(res) + res) on the bootstrapping parameter set at N = 2^12: the GPU
result equals the oracle running the same compiled program, bit for bit, and
decrypts to the input message (its real part for kImaginaryRemoving)."""
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
def _keys():
    o, g = pair(BOOT, LOGN)
    s = o.gen_secret(99, 32)
    return o, g, s, o.gen_mult_key(77, s), o.gen_conj_key(78, s)


@functools.lru_cache(maxsize=None)
def _rot_key(r):
    o, g, s, _, _ = _keys()
    return o.gen_rot_key(1000 + r, s, r)


@functools.lru_cache(maxsize=None)
def _setup(num_slots, variant):
    o, g, s, mk, ck = _keys()
    bc = chd.BootContext(g, num_slots=num_slots, variant=variant)
    rots = sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True)))
    rks = {r: _rot_key(r) for r in rots}
    keys = chd.EvkMap(g)
    keys.set_mult(g.evk(*mk))
    keys.set_conjugation(g.evk(*ck))
    for r, k in rks.items():
        keys.set_rotation(r, g.evk(*k))
    return bc, rks, keys


def _run(num_slots, variant, seed, min_ks=False):
    o, g, s, mk, ck = _keys()
    bc, rks, keys = _setup(num_slots, variant)
    rng = np.random.default_rng(seed)
    msg = (rng.random(num_slots) * 2 - 1) + 1j * (rng.random(num_slots) * 2 - 1)
    sc0 = o.scale(0)
    bx, ax = o.encrypt(seed, s, 0, o.encode(0, sc0, msg))
    res = bc.Boot(g.import_ct(0, [bx, ax], sc0, num_slots=num_slots), keys, min_ks=min_ks)
    parts = res.numpy()
    ref = run_program(o, bc.json(), Ct(0, [bx, ax], sc0), mult_key=mk, conj_key=ck, rot_keys=rks,
                      lts=bc.transforms(), min_ks=min_ks)
    assert ref.level == bc.end_level
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
    assert res.info()["num_slots"] == num_slots
    dec = o.decode(bc.end_level, bc.final_scale, o.decrypt(s, bc.end_level, parts), num_slots)
    return msg, dec, bc


@pytest.mark.parametrize("num_slots", [256, 1024])
def test_sparse_boot_bit_exact_and_precision(cuda_ok, num_slots):
    msg, dec, bc = _run(num_slots, chd.BOOT_NORMAL, 300 + num_slots)
    trace = [num_slots << i for i in range(20) if num_slots << i < 2048]
    assert set(trace) <= set(bc.rotations())
    err = np.abs(dec - msg).max()
    print(f"sparse bootstrapping, {num_slots} slots: {-np.log2(err):.2f} bits")
    assert -np.log2(err) > 10


def test_sparse_boot_min_ks(cuda_ok):
    msg, dec, _ = _run(512, chd.BOOT_NORMAL, 777, min_ks=True)
    assert -np.log2(np.abs(dec - msg).max()) > 10


@pytest.mark.parametrize("num_slots", [512, 2048])
def test_imaginary_removing(cuda_ok, num_slots):
    msg, dec, bc = _run(num_slots, chd.BOOT_IMAGINARY_REMOVING, 900 + num_slots)
    err = np.abs(dec - msg.real).max()
    print(f"kImaginaryRemoving, {num_slots} slots: {-np.log2(err):.2f} bits against the real part")
    assert -np.log2(err) > 10


def test_boot_slot_checks(cuda_ok):
    o, g, s, mk, ck = _keys()
    with pytest.raises(chd.CheddarError):
        chd.BootContext(g, num_slots=128)
    with pytest.raises(chd.CheddarError):
        chd.BootContext(g, num_slots=768)
    with pytest.raises(chd.CheddarError):
        chd.BootContext(g, num_slots=512, variant=3)
    bc, rks, keys = _setup(256, chd.BOOT_NORMAL)
    sc0 = o.scale(0)
    rng = np.random.default_rng(5)
    msg = rng.random(512) - 0.5
    bx, ax = o.encrypt(5, s, 0, o.encode(0, sc0, msg))
    with pytest.raises(chd.CheddarError):
        bc.Boot(g.import_ct(0, [bx, ax], sc0, num_slots=512), keys)


def test_merge_two_real(cuda_ok):
    # kMergeTwoReal: the StC constant is halved and nothing else changes
    # inside Boot (the caller merges two real inputs around it), so the
    # result decrypts to half the input
    msg, dec, _ = _run(512, chd.BOOT_MERGE_TWO_REAL, 4242)
    err = np.abs(dec - msg / 2).max()
    assert -np.log2(err) > 10


def test_sparse_boot_batch(cuda_ok):
    o, g, s, mk, ck = _keys()
    bc, rks, keys = _setup(512, chd.BOOT_NORMAL)
    sc0 = o.scale(0)
    rng = np.random.default_rng(8)
    cts = [o.encrypt(60 + i, s, 0, o.encode(0, sc0, rng.random(512) - 0.5)) for i in range(2)]
    single = [bc.Boot(g.import_ct(0, list(c), sc0, num_slots=512), keys).numpy() for c in cts]
    outs = bc.BootBatch([g.import_ct(0, list(c), sc0, num_slots=512) for c in cts], keys)
    for a, b in zip(outs, single):
        p = a.numpy()
        assert np.array_equal(p[0], b[0]) and np.array_equal(p[1], b[1])
