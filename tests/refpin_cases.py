"""Parity cases pinned to the reference's own code, one case per process.

Each case runs the reference's evaluator (oracle/_ref/libcheddar_ref.so: the
reference's src/core, src/extension and src/UserInterface.cu compiled for
sm_100a, driven through oracle/refdrv.py), this library (through its C ABI)
and, where it finishes in seconds, the CPU oracle on identical inputs, and
requires every residue to be equal.  The reference generates the secret, the
keys and the encryptions (its own client code, UserInterface.cu); they are
exported and imported into this library and the oracle.

One case per process because the reference keeps process-wide state per
parameter set (the ring degree, alpha and L in constant memory, written once
per process: include/common/ConstantMemory.cuh:16-33, NTT.cu:1226-1228), so
one process can only use one parameter set.  tests/test_gpu_refpin.py runs
every case as `python tests/refpin_cases.py <case>`; a case prints one JSON
line with its figures and exits 0, or raises.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "cheddar-fhe_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import cheddar_b200 as chd  # noqa: E402
import pyoracle as po  # noqa: E402
import refdrv  # noqa: E402

PARAMS = os.path.join(ROOT, "cheddar-fhe_b200", "params")


def load(name):
    return json.load(open(os.path.join(PARAMS, name)))


def ntt24_params():
    """The 24 main primes main_primes[2..25] of the reference's
    bootparam_30.json (all near 2^30, = 1 mod 2^17) as the q basis of a
    24-level chain, with its first 8 auxiliary primes."""
    b = load("bootparam_30.json")
    return {
        "log_degree": 16, "log_default_scale": 30, "boot": False,
        "dense_hamming_weight": 192, "sparse_hamming_weight": 32,
        "terminal_primes": [], "main_primes": b["main_primes"][2:26],
        "auxiliary_primes": b["auxiliary_primes"][:8],
        "default_encryption_level": 23,
        "level_config": [[i, 0] for i in range(1, 25)], "additional_base": [0, 0],
    }


def eq(what, got, want):
    got = [np.asarray(x) for x in got]
    want = [np.asarray(x) for x in want]
    assert len(got) == len(want), f"{what}: {len(got)} parts vs {len(want)}"
    for i, (a, b) in enumerate(zip(got, want)):
        assert a.shape == b.shape, f"{what}: part {i} shape {a.shape} vs {b.shape}"
        if not np.array_equal(a, b):
            bad = np.argwhere(a != b)
            raise AssertionError(f"{what}: part {i} differs at {len(bad)} words, first {bad[0].tolist()}")


def precision_bits(dec, msg):
    err = float(np.abs(np.asarray(dec) - np.asarray(msg)).max())
    return -float(np.log2(err)) if err > 0 else 99.0


def max_component_error(dec, msg):
    """Largest error of a real or imaginary part: the reference's test
    criterion is 1e-3 (unittest/Testbed.h:93, 318-322)."""
    d = np.asarray(dec) - np.asarray(msg)
    return float(max(np.abs(d.real).max(), np.abs(d.imag).max()))


class Trio:
    """The reference, this library and the oracle on one parameter set."""

    def __init__(self, params):
        self.p = params
        self.ref = refdrv.RefContext(params)
        self.g = chd.Context(json.dumps(params))
        self.o = po.Oracle(params)
        self.n = self.g.n
        self.keys = {}

    def key(self, idx):
        """(host (bx, ax), this library's EvaluationKey) of a reference key."""
        if idx not in self.keys:
            bx, ax, basis = self.ref.key(idx)
            self.keys[idx] = ((bx, ax), chd.EvaluationKey(self.g, bx, ax, basis=basis))
        return self.keys[idx]

    def rot_key(self, r):
        idx = r if r > 0 else self.n // 2 + r
        try:
            self.ref.key_shape(idx)
        except KeyError:
            self.ref.prepare_rotation(idx)
        return self.key(idx)

    def ct(self, rc):
        """A reference ciphertext as (host parts, this library's copy)."""
        inf = rc.info()
        parts = rc.numpy()
        level = self.level_of(inf)
        gc = self.g.import_ct(level, parts, scale=inf["scale"], num_slots=inf["num_slots"],
                              num_aux=inf["num_aux"])
        return parts, gc, level

    def level_of(self, inf):
        for lv in range(-1, self.g.max_level + 1):
            if self.g.level_np(lv) == (inf["num_main"], inf["num_ter"]):
                return lv
        raise AssertionError(f"no level holds {inf}")

    def message(self, seed, slots=None, lo=0.0, hi=1.0):
        rng = np.random.default_rng(seed)
        k = slots or self.n // 2
        return (rng.random(k) * (hi - lo) + lo) + 1j * (rng.random(k) * (hi - lo) + lo)


# ---------------------------------------------------------------- cases ----

def case_ntt24():
    """Forward NTT and inverse NTT of uniform residues over the 24 primes
    main_primes[2..25] of bootparam_30.json: NTTHandler::NTT(..., false) and
    INTT(..., true) (NTT.cu:606-741) against this library's raw transforms
    and the oracle; the round trip returns the input."""
    import torch
    t = Trio(ntt24_params())
    lvl = 23
    m, _ = t.g.level_np(lvl)
    assert m == 24
    rng = np.random.default_rng(0)
    q = np.array(t.p["main_primes"], dtype=np.uint64)[:, None]
    x = (rng.integers(0, 2 ** 62, size=(2, 24, t.n), dtype=np.uint64) % q).astype(np.uint32)
    # edge values in the first columns
    x[:, :, 0] = 0
    x[:, :, 1] = (q[:, 0] - 1).astype(np.uint32)
    ref_f = t.ref.ntt(24, 0, 0, x, inverse=False, montgomery=False)
    dev = torch.from_numpy(x.view(np.int32).copy()).cuda()
    t.g.ntt_raw(24, 0, 0, dev, mont=False, count=2)
    t.g.synchronize()
    ours_f = dev.cpu().numpy().view(np.uint32)
    orc_f = np.stack([t.o.ntt(lvl, x[i]) for i in range(2)])
    eq("NTT vs reference", [ours_f], [ref_f])
    eq("NTT vs oracle", [ours_f], [orc_f])
    # INTT(..., true) also leaves the Montgomery domain (x 2^-32)
    ref_i = t.ref.ntt(24, 0, 0, ref_f, inverse=True, montgomery=True)
    t.g.intt_raw(24, 0, 0, dev, mont=True, count=2)
    t.g.synchronize()
    ours_i = dev.cpu().numpy().view(np.uint32)
    eq("INTT vs reference", [ours_i], [ref_i])
    eq("INTT vs oracle", [ours_i], [np.stack([t.o.intt(lvl, ref_f[i]) for i in range(2)])])
    # Montgomery-converting forward transform (NTT(..., true), x 2^32), whose
    # inverse INTT(..., true) returns the input
    ref_fm = t.ref.ntt(24, 0, 0, x, inverse=False, montgomery=True)
    dev = torch.from_numpy(x.view(np.int32).copy()).cuda()
    t.g.ntt_raw(24, 0, 0, dev, mont=True, count=2)
    t.g.synchronize()
    eq("NTT(mont) vs reference", [dev.cpu().numpy().view(np.uint32)], [ref_fm])
    t.g.intt_raw(24, 0, 0, dev, mont=True, count=2)
    t.g.synchronize()
    eq("round trip", [dev.cpu().numpy().view(np.uint32)], [x])
    eq("reference round trip", [t.ref.ntt(24, 0, 0, ref_fm, inverse=True, montgomery=True)], [x])
    return {"primes": 24, "polys": 2}


def case_modswitch():
    """ModUp, ModDown, Rescale and ModDownAndRescale (ModSwitch.cu:429-684)
    at several levels of the L = 24, alpha = 8 key-switching set, on uniform
    residues: reference, this library and the oracle."""
    import torch
    t = Trio(load("keyswitch_l24_a8.json"))
    o, g = t.o, t.g
    levels = [22, 21, 15, 8, 1]
    for lvl in levels:
        x = o.uniform(10 + lvl, lvl)
        ref_mu = t.ref.modup(lvl, x)
        mu = torch.zeros((o.beta(lvl), o.num_q(lvl) + o.alpha, o.n), dtype=torch.int32, device="cuda")
        g.modup_raw(lvl, torch.from_numpy(x.view(np.int32)).cuda(), mu)
        g.synchronize()
        ours_mu = mu.cpu().numpy().view(np.uint32).reshape(ref_mu.shape)
        eq(f"ModUp level {lvl} vs reference", [ours_mu], [ref_mu])
        eq(f"ModUp level {lvl} vs oracle", [ours_mu], [o.modup(lvl, x)])
        xa = o.uniform(20 + lvl, lvl, num_aux=o.alpha)
        out = torch.zeros((o.num_q(lvl), o.n), dtype=torch.int32, device="cuda")
        g.moddown_raw(lvl, chd.CHD_MODDOWN, torch.from_numpy(xa.view(np.int32)).cuda(), out)
        g.synchronize()
        eq(f"ModDown level {lvl}", [out.cpu().numpy().view(np.uint32)], [t.ref.moddown(lvl, 0, xa)])
        out1 = torch.zeros((o.num_q(lvl - 1), o.n), dtype=torch.int32, device="cuda")
        g.moddown_raw(lvl, chd.CHD_RESCALE, torch.from_numpy(x.view(np.int32)).cuda(), out1)
        g.synchronize()
        eq(f"Rescale level {lvl}", [out1.cpu().numpy().view(np.uint32)], [t.ref.moddown(lvl, 1, x)])
        g.moddown_raw(lvl, chd.CHD_MODDOWN_RESCALE, torch.from_numpy(xa.view(np.int32)).cuda(), out1)
        g.synchronize()
        eq(f"ModDownAndRescale level {lvl}", [out1.cpu().numpy().view(np.uint32)], [t.ref.moddown(lvl, 2, xa)])
    return {"levels": levels}


def case_keyswitch():
    """HMult (+ relinearize + rescale), HMult without rescale, HRot (several
    offsets, negative ones included), HConj and Rescale at several levels of
    the L = 24, alpha = 8 set, on the reference's own keys and encryptions:
    Context::HMult / HRot / HConj (Context.cpp:776-871) against this library
    and the oracle; decoded precision of the product by the reference's own
    decryption and decoder."""
    t = Trio(load("keyswitch_l24_a8.json"))
    o, g, ref = t.o, t.g, t.ref
    (mkb, mka), mk = t.key(ref.MULT)
    (ckb, cka), ck = t.key(ref.CONJ)
    out = {"levels": {}}
    for lvl, seed in [(22, 1), (21, 2), (12, 3), (3, 4), (1, 5)]:
        m1, m2 = t.message(seed), t.message(seed + 100)
        ra, rb = ref.encrypt(lvl, m1), ref.encrypt(lvl, m2)
        pa, ga, la = t.ct(ra)
        pb, gb, _ = t.ct(rb)
        assert la == lvl
        r_ref = ref.HMult(ra, rb, rescale=True)
        r_g = g.HMult(ga, gb, mk, rescale=True)
        eq(f"HMult level {lvl} vs reference", r_g.numpy(), r_ref.numpy())
        eq(f"HMult level {lvl} vs oracle", r_g.numpy(), o.hmult(lvl, pa, pb, (mkb, mka), rescale=True))
        dec = ref.decrypt_decode(r_ref)
        bits = precision_bits(dec, m1 * m2)
        assert bits > 10, bits
        r_ref2 = ref.HMult(ra, rb, rescale=False)
        eq(f"HMult no rescale level {lvl}", g.HMult(ga, gb, mk, rescale=False).numpy(), r_ref2.numpy())
        eq(f"Rescale level {lvl}", g.Rescale(g.HMult(ga, gb, mk, rescale=False)).numpy(),
           ref.Rescale(r_ref2).numpy())
        for rot in ([1, 5, -1, 1 << 10, t.n // 2 - 1] if lvl in (22, 3) else [3]):
            (kb, ka), rk = t.rot_key(rot)
            h_ref = ref.HRot(ra, rot)
            h_g = g.HRot(ga, rk, rot)
            eq(f"HRot {rot} level {lvl} vs reference", h_g.numpy(), h_ref.numpy())
            eq(f"HRot {rot} level {lvl} vs oracle", h_g.numpy(), o.hrot(lvl, pa, (kb, ka), rot % (t.n // 2)))
        c_ref = ref.HConj(ra)
        eq(f"HConj level {lvl} vs reference", g.HConj(ga, ck).numpy(), c_ref.numpy())
        eq(f"HConj level {lvl} vs oracle", g.HConj(ga, ck).numpy(), o.hconj(lvl, pa, (ckb, cka)))
        out["levels"][lvl] = {"hmult_precision_bits": round(bits, 2)}
    return out


def case_mixed_batch():
    """One HMultBatch call over the reference's encryptions at ten different
    levels of the L = 24, alpha = 8 set (this library runs them as one fused
    pipeline, the row pass taking several levels per launch) against one
    Context::HMult call of the reference per pair (Context.cpp:862-871),
    with and without rescale."""
    t = Trio(load("keyswitch_l24_a8.json"))
    g, ref = t.g, t.ref
    _, mk = t.key(ref.MULT)
    levels = [22, 3, 17, 9, 1, 20, 12, 5, 14, 7]
    ras, rbs, gas, gbs = [], [], [], []
    for i, lvl in enumerate(levels):
        ra, rb = ref.encrypt(lvl, t.message(300 + i)), ref.encrypt(lvl, t.message(400 + i))
        ras.append(ra)
        rbs.append(rb)
        gas.append(t.ct(ra)[1])
        gbs.append(t.ct(rb)[1])
    for rescale in (True, False):
        outs = g.HMultBatch(gas, gbs, mk, rescale=rescale)
        for lvl, ra, rb, r in zip(levels, ras, rbs, outs):
            eq(f"HMultBatch level {lvl} rescale {rescale}", r.numpy(), ref.HMult(ra, rb, rescale=rescale).numpy())
    return {"levels": levels, "pairs": len(levels)}


def case_w64():
    """The 64-bit word path against the reference's own Context<uint64_t>
    on its bootparam_40_64bit.json (40-55-bit main primes, 56-bit auxiliary
    primes, alpha = 7): NTT / INTT with and without the Montgomery
    conversion (NTT.cu:606-741), ModUp, ModDown, Rescale and
    ModDownAndRescale (ModSwitch.cu:429-684) at several levels, HMult with
    and without rescale, HRot and HConj (Context.cpp:776-871) on uniform
    ciphertexts and uniform keys (both are deterministic functions of their
    inputs), every word equal."""
    import torch
    p = load("bootparam_40_64bit.json")
    ref = refdrv.RefContext64(p)
    g = chd.Context64(json.dumps(p))
    n = g.n
    primes = g.primes()
    nt, nm, na = len(p["terminal_primes"]), len(p["main_primes"]), len(p["auxiliary_primes"])
    L = nt + nm
    rng = np.random.default_rng(64)

    def rows_of(level, aux):
        m, t = g.level_np(level)
        return [nt - t + i for i in range(m + t)] + [L + a for a in range(aux)]

    def uniform(rows):
        return np.stack([rng.integers(0, int(primes[r]), n, dtype=np.uint64) for r in rows])

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
        torch.cuda.synchronize()  # the context works on its own stream
        return t

    def host(t):
        torch.cuda.synchronize()
        return t.cpu().numpy().view(np.uint64)

    out = {"params": "bootparam_40_64bit.json", "levels": []}
    # NTT / INTT over the top level with the auxiliary primes
    m, t = g.level_np(g.max_level)
    x = np.stack([uniform(rows_of(g.max_level, na)) for _ in range(2)])
    for inverse in (False, True):
        for mont in (False, True):
            d = dev(x)
            g.ntt((m, t, na), d, count=2, inverse=inverse, mont=mont)
            g.synchronize()
            eq(f"64-bit {'INTT' if inverse else 'NTT'} mont={mont}", host(d).reshape(x.shape),
               ref.ntt((m, t, na), x, inverse=inverse, mont=mont))
    beta_max = -(-L // na)
    kb = np.stack([uniform(rows_of(g.max_level, na)) for _ in range(beta_max)])
    ka = np.stack([uniform(rows_of(g.max_level, na)) for _ in range(beta_max)])
    key = chd.EvaluationKey64(g, kb, ka)
    for lvl in (g.max_level, 17, 9, 3, 1):
        m, t = g.level_np(lvl)
        q = m + t
        beta = -(-q // na)
        src = uniform(rows_of(lvl, 0))
        mu = torch.zeros((beta, q + na, n), dtype=torch.int64, device="cuda")
        g.modup_raw(lvl, dev(src), mu)
        g.synchronize()
        eq(f"64-bit ModUp level {lvl}", host(mu), ref.modup(lvl, src, beta, q + na))
        xa = uniform(rows_of(lvl, na))
        o = torch.zeros((q, n), dtype=torch.int64, device="cuda")
        g.moddown_raw(lvl, chd.CHD_MODDOWN, dev(xa), o)
        g.synchronize()
        eq(f"64-bit ModDown level {lvl}", host(o), ref.moddown(lvl, 0, xa, q))
        mq = sum(g.level_np(lvl - 1))
        o1 = torch.zeros((mq, n), dtype=torch.int64, device="cuda")
        g.moddown_raw(lvl, chd.CHD_RESCALE, dev(src), o1)
        g.synchronize()
        eq(f"64-bit Rescale level {lvl}", host(o1), ref.moddown(lvl, 1, src, mq))
        g.moddown_raw(lvl, chd.CHD_MODDOWN_RESCALE, dev(xa), o1)
        g.synchronize()
        eq(f"64-bit ModDownAndRescale level {lvl}", host(o1), ref.moddown(lvl, 2, xa, mq))
        a = (uniform(rows_of(lvl, 0)), uniform(rows_of(lvl, 0)))
        b = (uniform(rows_of(lvl, 0)), uniform(rows_of(lvl, 0)))
        ga, gb = g.import_ct(lvl, a), g.import_ct(lvl, b)
        for rescale in (True, False):
            rows_out = mq if rescale else q
            eq(f"64-bit HMult level {lvl} rescale {rescale}", g.HMult(ga, gb, key, rescale).numpy(),
               ref.hmult(lvl, a, b, (kb, ka), rescale, rows_out))
        for rot in ((1, 5, n // 2 - 1) if lvl in (g.max_level, 3) else (2,)):
            eq(f"64-bit HRot {rot} level {lvl}", g.HRot(ga, key, rot).numpy(), ref.hrot(lvl, a, (kb, ka), rot, q))
        eq(f"64-bit HConj level {lvl}", g.HConj(ga, key).numpy(), ref.hconj(lvl, a, (kb, ka), q))
        out["levels"].append(lvl)
    return out


def case_w64_ops():
    """The 64-bit word path's Context operations against the reference's
    own Context<uint64_t> on bootparam_40_64bit.json (Context.h:101-423):
    Copy, Neg, MultImaginaryUnit, Add / Sub (also with rx on one side),
    Mult (three-part tensor), Relinearize, RelinearizeRescale, MultKey,
    Permute, PermuteConjugate, HRotAdd, HConjAdd, MultConst / AddConst
    (constants from each side's own EncodeConstant) and LevelDown, on
    uniform ciphertexts and keys at several levels, every word equal."""
    p = load("bootparam_40_64bit.json")
    ref = refdrv.RefContext64(p)
    g = chd.Context64(json.dumps(p))
    n = g.n
    primes = g.primes()
    nt, nm, na = len(p["terminal_primes"]), len(p["main_primes"]), len(p["auxiliary_primes"])
    L = nt + nm
    rng = np.random.default_rng(640)

    def rows_of(level, aux=0):
        m, t = g.level_np(level)
        return [nt - t + i for i in range(m + t)] + [L + a for a in range(aux)]

    def uniform(rows):
        return np.stack([rng.integers(0, int(primes[r]), n, dtype=np.uint64) for r in rows])

    beta_max = -(-L // na)
    kb = np.stack([uniform(rows_of(g.max_level, na)) for _ in range(beta_max)])
    ka = np.stack([uniform(rows_of(g.max_level, na)) for _ in range(beta_max)])
    key = chd.EvaluationKey64(g, kb, ka)
    K = (kb, ka)
    enc = p["default_encryption_level"]
    checked = []
    for lvl in sorted({g.max_level, enc, 9, 2}, reverse=True):
        scale = g.scale(min(lvl, enc))  # the imported ciphertexts' scale
        a = tuple(uniform(rows_of(lvl)) for _ in range(2))
        b = tuple(uniform(rows_of(lvl)) for _ in range(2))
        r3 = uniform(rows_of(lvl))
        ga, gb = g.import_ct(lvl, a, scale=scale), g.import_ct(lvl, b, scale=scale)
        g3 = g.import_ct(lvl, a, scale=scale).set_rx(r3)
        a3 = a + (r3,)
        cx = g.encode_const(lvl, scale, 0.6180339887)
        pairs = [
            ("Copy", g.Copy(ga), ref.op("Copy", lvl, a)),
            ("Neg", g.Neg(ga), ref.op("Neg", lvl, a)),
            ("Neg rx", g.Neg(g3), ref.op("Neg", lvl, a3)),
            ("MultImaginaryUnit", g.MultImaginaryUnit(ga), ref.op("MultImaginaryUnit", lvl, a)),
            ("Add", g.Add(ga, gb), ref.op("Add", lvl, a, b)),
            ("Sub", g.Sub(ga, gb), ref.op("Sub", lvl, a, b)),
            ("Add rx", g.Add(g3, gb), ref.op("Add", lvl, a3, b)),
            ("Sub rx", g.Sub(gb, g3), ref.op("Sub", lvl, b, a3)),
            ("Mult", g.Mult(ga, gb), ref.op("Mult", lvl, a, b)),
            ("Relinearize", g.Relinearize(g3, key), ref.op("Relinearize", lvl, a3, key=K)),
            ("MultKey", g.MultKey(ga, key), ref.op("MultKey", lvl, a, key=K)),
            ("Permute", g.Permute(ga, 5), ref.op("Permute", lvl, a, arg=5)),
            ("PermuteConjugate", g.PermuteConjugate(ga), ref.op("PermuteConjugate", lvl, a)),
            ("HRotAdd", g.HRotAdd(ga, gb, key, 3), ref.op("HRotAdd", lvl, a, b, key=K, arg=3)),
            ("HConjAdd", g.HConjAdd(ga, gb, key), ref.op("HConjAdd", lvl, a, b, key=K)),
            ("MultConst", g.MultConst(ga, cx, scale), ref.op("MultConst", lvl, a, scale=scale, value=0.6180339887)),
            ("AddConst", g.AddConst(ga, cx), ref.op("AddConst", lvl, a, scale=scale, value=0.6180339887)),
        ]
        if lvl >= 1:
            pairs.append(("RelinearizeRescale", g.RelinearizeRescale(g3, key),
                          ref.op("RelinearizeRescale", lvl, a3, key=K)))
        if 2 <= lvl <= enc:
            pairs.append(("LevelDown", g.LevelDown(ga, lvl - 2), ref.op("LevelDown", lvl, a, arg=lvl - 2)))
        for what, ours, theirs in pairs:
            mine = ours.numpy()
            assert len(mine) == len(theirs), f"64-bit {what} level {lvl}: parts {len(mine)} vs {len(theirs)}"
            eq(f"64-bit {what} level {lvl}", list(mine), list(theirs))
            checked.append(f"{what}@{lvl}")
    return {"params": "bootparam_40_64bit.json", "checked": len(checked)}


def case_hoisted():
    """Hoisted rotations: the reference's HoistHandler::EvaluateBabyStep
    (Hoist.cu:578-691; one ModUp, every rotation's key product and
    automorphism in one fused launch, results in basis Q u P) for the 30
    offsets +-2^k (k < 15) and 1..4 at the top level of the L = 24 set,
    against this library's hoisted rotation and the oracle."""
    t = Trio(load("keyswitch_l24_a8.json"))
    o, g, ref = t.o, t.g, t.ref
    half = t.n // 2
    offs = sorted({(s * (1 << k)) % half for k in range(15) for s in (1, -1)} | {1, 2, 3, 4})
    assert len(offs) == 30
    lvl = g.max_level
    ra = ref.encrypt(lvl, t.message(7))
    pa, ga, _ = t.ct(ra)
    keys = [t.rot_key(r) for r in offs]
    bs_ref = ref.hoisted_baby_steps(ra, offs)
    outs = g.HoistedRotate(ga, [k[1] for k in keys], offs)
    hb, ha = o.hoisted_rotate(lvl, pa, [k[0] for k in keys], offs)
    for i, r in enumerate(offs):
        eq(f"baby step {r} vs reference", outs[i].numpy(), bs_ref[i].numpy())
        eq(f"baby step {r} vs oracle", outs[i].numpy(), [hb[i], ha[i]])
    return {"offsets": len(offs), "level": lvl}


def case_encode():
    """Encoder::Encode (Encode.cpp:135-190: special IFFT, scaling, truncation
    to an integer, residues, NTT) of the reference against this library's
    encoder, at several levels, scales and aux counts of bootparam_40.json."""
    t = Trio(load("bootparam_40.json"))
    g, ref = t.g, t.ref
    cases = 0
    for lvl, num_aux, seed in [(0, 0, 1), (5, 0, 2), (16, 12, 3), (28, 12, 4), (13, 0, 5)]:
        msg = t.message(seed, lo=-1.0, hi=1.0)
        for sc in (ref.test_scale(lvl), 2.0 ** 40, 2.0 ** 52):
            got = g.encode(lvl, sc, msg, num_aux=num_aux)
            g.synchronize()
            got = got.cpu().numpy().view(np.uint32)
            want = ref.encode(lvl, sc, msg, num_aux=num_aux)
            eq(f"Encode level {lvl} aux {num_aux} scale 2^{np.log2(sc):.2f}", [got], [want])
            cases += 1
    return {"cases": cases}


def _context_ops(name, levels):
    """Add, Sub, Neg, Mult (three-part tensor), Relinearize,
    RelinearizeRescale, Rescale, MultKey, Permute, PermuteConjugate,
    MultImaginaryUnit, LevelDown, HRotAdd, HConjAdd, MultUnsafe and HMult
    (Context.cpp:316-949) on the reference's encryptions and keys, against
    this library."""
    t = Trio(load(name))
    g, ref = t.g, t.ref
    mk = t.key(ref.MULT)[1]
    ck = t.key(ref.CONJ)[1]
    checked = []
    for lvl, seed in levels:
        ra, rb = ref.encrypt(lvl, t.message(seed)), ref.encrypt(lvl, t.message(seed + 50))
        _, ga, _ = t.ct(ra)
        _, gb, _ = t.ct(rb)
        rot = 3
        rk = t.rot_key(rot)[1]
        pairs = [
            ("Add", g.Add(ga, gb), ref.binary("Add", ra, rb)),
            ("Sub", g.Sub(ga, gb), ref.binary("Sub", ra, rb)),
            ("Neg", g.Neg(ga), ref.unary("Neg", ra)),
            ("MultImaginaryUnit", g.MultImaginaryUnit(ga), ref.unary("MultImaginaryUnit", ra)),
            ("Copy", g.Copy(ga), ref.unary("Copy", ra)),
            ("HMult", g.HMult(ga, gb, mk), ref.HMult(ra, rb)),
            ("HRotAdd", g.HRotAdd(ga, gb, rk, rot), ref.binary("HRotAdd", ra, rb, rot)),
            ("HConjAdd", g.HConjAdd(ga, gb, ck), ref.binary("HConjAdd", ra, rb)),
            ("MultKey", g.MultKey(ga, rk), ref.unary("MultKeyRot", ra, rot)),
        ]
        gm, rm = g.Mult(ga, gb), ref.binary("Mult", ra, rb)
        pairs += [("Mult", gm, rm),
                  ("Relinearize", g.Relinearize(gm, mk), ref.unary("Relinearize", rm)),
                  ("RelinearizeRescale", g.RelinearizeRescale(gm, mk), ref.unary("RelinearizeRescale", rm))]
        gr, rr = g.Relinearize(gm, mk), ref.unary("Relinearize", rm)
        pairs += [("Rescale", g.Rescale(gr), ref.Rescale(rr)),
                  ("Permute", g.Permute(g.MultKey(ga, rk), rot), ref.unary("Permute", ref.unary("MultKeyRot", ra, rot),
                                                                         rot))]
        # the reference's level-down constants exist up to the default
        # encryption level (Context.cpp:102-107); above it LevelDown reads
        # past them, so it is compared only where it is defined
        if 2 <= lvl <= t.p["default_encryption_level"]:
            pairs.append(("LevelDown", g.LevelDown(ga, lvl - 2), ref.unary("LevelDown", ra, lvl - 2)))
        if lvl >= 1 and g.IsMultUnsafeCompatible(lvl, lvl - 1):
            pairs.append(("MultUnsafe", g.MultUnsafe(ga, gb, lvl - 1), ref.binary("MultUnsafe", ra, rb, lvl - 1)))
        for what, ours, theirs in pairs:
            eq(f"{what} level {lvl}", ours.numpy(), theirs.numpy())
            checked.append(f"{what}@{lvl}")
    return {"params": name, "checked": len(checked)}


def case_context_ops():
    return _context_ops("keyswitch_l24_a8.json", [(22, 1), (10, 2), (1, 3)])


def case_context_ops40():
    """The same on bootparam_40.json, whose low levels mix main and terminal
    primes (rational rescale, ModDown with terminal-prime restore)."""
    return _context_ops("bootparam_40.json", [(28, 1), (16, 2), (5, 3), (4, 4), (3, 5), (2, 6), (1, 7)])


def case_decode():
    """Encoder::Decode (Encode.cpp:45-70, 192-248) of the reference against
    this library's device decoder, double for double: plaintexts the
    reference decrypts from its own encryptions (at several levels and slot
    counts of bootparam_40.json, terminal primes included) and from products
    (HMult), and plaintexts of the library's encoder."""
    import torch
    t = Trio(load("bootparam_40.json"))
    g, ref = t.g, t.ref
    checked = 0
    for lvl, ns, seed in [(0, t.n // 2, 1), (3, 1 << 10, 2), (13, t.n // 2, 3), (16, 256, 4), (28, t.n // 2, 5)]:
        msg = t.message(seed, slots=ns, lo=-1.0, hi=1.0)
        pt, sc, nsl = ref.decrypt(ref.encrypt(lvl, msg))
        assert nsl == ns
        want = ref.decode(lvl, sc, ns, pt)
        got = g.decode(lvl, sc, torch.from_numpy(pt.view(np.int32)).cuda(), ns)
        assert np.array_equal(got, want), f"decode level {lvl}: max diff {np.abs(got - want).max()}"
        assert max_component_error(got, msg) < 1e-3
        checked += 1
        enc = g.encode(lvl, ref.test_scale(lvl), msg)
        g.synchronize()
        pt2 = enc.cpu().numpy().view(np.uint32)
        want = ref.decode(lvl, ref.test_scale(lvl), ns, pt2)
        got = g.decode(lvl, ref.test_scale(lvl), enc, ns)
        assert np.array_equal(got, want), f"decode of an encoding, level {lvl}"
        checked += 1
    lvl = 16
    ra, rb = ref.encrypt(lvl, t.message(9)), ref.encrypt(lvl, t.message(10))
    pt, sc, ns = ref.decrypt(ref.HMult(ra, rb))
    want = ref.decode(lvl - 1, sc, ns, pt)
    got = g.decode(lvl - 1, sc, torch.from_numpy(pt.view(np.int32)).cuda(), ns)
    assert np.array_equal(got, want), "decode of a product"
    return {"checked": checked + 1}


def _boot_trio(name, num_slots=None):
    t = Trio(load(name))
    g, ref = t.g, t.ref
    ns = num_slots or t.n // 2
    rots = ref.boot_prepare(ns)
    bc = chd.BootContext(g, num_slots=ns)
    ours = sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True)))
    assert sorted(rots) == ours, f"rotation sets differ: reference {sorted(rots)} vs {ours}"
    keys = chd.EvkMap(g)
    keys.set_mult(t.key(ref.MULT)[1])
    keys.set_conjugation(t.key(ref.CONJ)[1])
    for r in rots:
        keys.set_rotation(r, t.key(r)[1])
    if t.p["dense_hamming_weight"] != t.p["sparse_hamming_weight"]:
        bx, ax, basis = ref.key(ref.DTS)
        dts = chd.EvaluationKey(g, bx, ax, basis=basis)
        bx, ax, basis = ref.key(ref.STD)
        # the sparse-to-dense key's digits are summed into digit 0
        # (UserInterface.cu:341-351); only that digit is used
        std = chd.EvaluationKey(g, bx[:1], ax[:1], basis=basis)
        t.keys["dts"], t.keys["std"] = (None, dts), (None, std)
        keys.set_dense_to_sparse(dts)
        keys.set_sparse_to_dense(std)
    return t, bc, keys, rots


def _boot_case(name, num_slots=None, min_bits=18.5):
    """BootContext::Boot (BootContext.cpp:299-365, hoisted and min-KS) of
    the reference against this library's Boot and BootBatch on the
    reference's keys and its encryption of uniform slots in [-1, 1]^2 at
    level 0; decoded precision by the reference's own decryption and
    decoder (the two outputs are the same residues, hence the same
    precision)."""
    t, bc, keys, rots = _boot_trio(name, num_slots)
    ref, g = t.ref, t.g
    ns = num_slots or t.n // 2
    msgs = [t.message(11 + i, slots=ns, lo=-1.0, hi=1.0) for i in range(2)]
    rin = [ref.encrypt(0, m) for m in msgs]
    gin = [t.ct(r)[1] for r in rin]
    res = {"params": name, "slots": ns, "rotations": len(rots)}
    for min_ks in (False, True):
        tag = "min-KS" if min_ks else "hoisted"
        r_ref = ref.Boot(rin[0], min_ks=min_ks)
        r_g = bc.Boot(gin[0], keys, min_ks=min_ks)
        eq(f"Boot ({tag}) vs reference", r_g.numpy(), r_ref.numpy())
        batch = bc.BootBatch(gin, keys, min_ks=min_ks)
        eq(f"BootBatch[0] ({tag}) vs reference", batch[0].numpy(), r_ref.numpy())
        r_ref1 = ref.Boot(rin[1], min_ks=min_ks)
        eq(f"BootBatch[1] ({tag}) vs reference", batch[1].numpy(), r_ref1.numpy())
        inf = r_ref.info()
        d0, d1 = ref.decrypt_decode(r_ref), ref.decrypt_decode(r_ref1)
        bits = min(precision_bits(d0, msgs[0]), precision_bits(d1, msgs[1]))
        comp = max(max_component_error(d0, msgs[0]), max_component_error(d1, msgs[1]))
        res[tag] = {"precision_bits": round(bits, 2), "max_component_error": comp, "end_level": t.level_of(inf),
                    "end_scale_log2": round(float(np.log2(inf["scale"])), 4)}
        assert comp <= 1e-3, (tag, comp)
        assert bits >= min_bits, (tag, bits)
    return res


def case_boot40():
    """Full-slot bootstrapping at N = 2^16 on the reference's own
    bootparam_40.json (4 terminal + 43 main primes, alpha = 12, sparse-secret
    encapsulation)."""
    return _boot_case("bootparam_40.json")


def case_boot30():
    """Full-slot bootstrapping on bootparam_30.json (48 main primes, no
    terminal primes)."""
    return _boot_case("bootparam_30.json", min_bits=9.9)


def case_boot35():
    """Full-slot bootstrapping on bootparam_35.json (5 terminal primes)."""
    return _boot_case("bootparam_35.json", min_bits=9.9)


def case_boot40_sparse():
    """Bootstrapping of 2^10 slots (sparse packing: Trace, the 2n x 2n
    CoeffToSlot / SlotToCoeff phases) on bootparam_40.json."""
    return _boot_case("bootparam_40.json", num_slots=1 << 10, min_bits=9.9)


CASES = {k[5:]: v for k, v in globals().items() if k.startswith("case_")}


def main(argv):
    name = argv[1]
    out = CASES[name]()
    print(json.dumps({"case": name, **out}), flush=True)
    # Skip interpreter teardown: the reference's objects hold device memory
    # from its process-wide pool, and module teardown order is arbitrary.
    os._exit(0)


if __name__ == "__main__":
    main(sys.argv)
