"""CPU restatement of the reference's bootstrapping evaluation steps, built on
the C oracle's primitives (test infrastructure: used only by tests/ and the
bench's CPU baseline; never by the product path).

Linear transforms: HoistHandler::Evaluate with the fused baby-step and
giant-step kernels (src/extension/Hoist.cu:21-118, 207-420, 554-975), for a
compiled plaintext map [(giant step, baby step, message)].  The modular
arithmetic is done with numpy on canonical residues (Montgomery products as
a*b*2^-32 mod q), so every value is the unique canonical residue the
reference's kernels produce.
"""
import numpy as np

_RINV = {}


def _rinv(q):
    q = int(q)
    if q not in _RINV:
        _RINV[q] = pow(2 ** 32, -1, q)
    return _RINV[q]


def mont_mul(a, b, q):
    """Canonical a * b * 2^-32 mod q (basic::MultMontgomery)."""
    q = np.uint64(q)
    x = (np.asarray(a, dtype=np.uint64) * np.asarray(b, dtype=np.uint64)) % q
    return ((x * np.uint64(_rinv(int(q)))) % q).astype(np.uint32)


def add_mod(a, b, q):
    q = np.uint64(q)
    return ((np.asarray(a, dtype=np.uint64) + np.asarray(b, dtype=np.uint64)) % q).astype(np.uint32)


class HoistOracle:
    """One (oracle, level) pair: the Q u P basis of `level` and its constants."""

    def __init__(self, o, level):
        self.o = o
        self.level = level
        self.nq = o.num_q(level)
        self.alpha = o.alpha
        self.tot = self.nq + self.alpha
        self.primes = [int(p) for p in o.primes(level, self.alpha)]
        m, t = o.level_np(level)
        self.max_ter = len(o.params.get("terminal_primes", []))
        self.prime_offset = self.max_ter - t
        L = self.max_ter + len(o.params["main_primes"])
        self.L = L
        aux = [int(p) for p in o.params["auxiliary_primes"]][: self.alpha]
        # P mod q in Montgomery form (Context.cpp:78-90)
        self.p_prod = []
        for q in self.primes[: self.nq]:
            v = 1
            for a in aux:
                v = v * a % q
            self.p_prod.append(v * (2 ** 32) % q)
        self.beta = o.beta(level)

    def zeros(self):
        return np.zeros((self.tot, self.o.n), dtype=np.uint32)

    def pseudo_modup(self, x):
        """PseudoModUp + ZeroExtend: P * x on the q rows, 0 on the aux rows."""
        out = self.zeros()
        for r in range(self.nq):
            out[r] = mont_mul(x[r], self.p_prod[r], self.primes[r])
        return out

    def pmul(self, x, pt):
        out = self.zeros()
        for r in range(self.tot):
            out[r] = mont_mul(x[r], pt[r], self.primes[r])
        return out

    def add(self, x, y, rows=None):
        out = np.array(x, copy=True)
        for r in range(self.tot if rows is None else rows):
            out[r] = add_mod(x[r], y[r], self.primes[r])
        return out

    def key_mult(self, mu, key):
        """MultKeyNoModDown (Context.cpp:610-648): sum_i mu_i (.) key_i."""
        kb, ka = key
        ob, oa = self.zeros(), self.zeros()
        padded = self.nq + self.prime_offset
        for i in range(self.beta):
            if min((i + 1) * self.alpha, padded) <= self.prime_offset:
                continue
            for r in range(self.tot):
                kr = self.prime_offset + r if r < self.nq else self.L + (r - self.nq)
                q = self.primes[r]
                ob[r] = add_mod(ob[r], mont_mul(mu[i][r], kb[i][kr], q), q)
                oa[r] = add_mod(oa[r], mont_mul(mu[i][r], ka[i][kr], q), q)
        return ob, oa

    def permute(self, x, amount):
        return self.o.permute(self.level, amount, x, num_aux=self.alpha)


def _stride(idx):
    """HoistHandler::CheckStrideMinKS (Hoist.cu:169-205)."""
    import math
    g, cnt, mx = 0, 0, 0
    for x in idx:
        if x:
            g = math.gcd(g, x)
            cnt += 1
            mx = max(mx, x)
    assert cnt * g == mx, "MinKS does not apply to the given sequence"
    return g


def lt_evaluate(o, level, ct, ct_scale, pts, pt_scale, keys, min_ks=False):
    """HoistHandler::Evaluate for the compiled map `pts` = [(gs, bs, msg)];
    keys = {rotation: (kb, ka)}.  Returns ((bx, ax) at level - 1, scale)."""
    h = HoistOracle(o, level)
    bx, ax = ct
    enc = {(g, b): o.encode(level, pt_scale, m, num_aux=h.alpha) for g, b, m in pts}
    bs_set = sorted({b for _, b, _ in pts})
    gs_set = sorted({g for g, _, _ in pts})
    if min_ks:
        # EvaluateMinKSBabyStep / EvaluateMinKSGiantStep (Hoist.cu:490-552)
        nq = h.nq
        bstr, gstr = _stride(bs_set), _stride(gs_set)
        bs = {}
        for b in bs_set:
            if b == 0:
                bs[0] = (np.asarray(bx), np.asarray(ax))
            else:
                bs[b] = o.hrot(level, bs[b - bstr], keys[bstr], bstr)
        acc = None
        for g in reversed(gs_set):
            sb = np.zeros((nq, o.n), dtype=np.uint32)
            sa = np.zeros_like(sb)
            for b in bs_set:
                if (g, b) not in enc:
                    continue
                pt = enc[(g, b)]
                for r in range(nq):
                    q = h.primes[r]
                    sb[r] = add_mod(sb[r], mont_mul(bs[b][0][r], pt[r], q), q)
                    sa[r] = add_mod(sa[r], mont_mul(bs[b][1][r], pt[r], q), q)
            if acc is not None:
                for r in range(nq):
                    q = h.primes[r]
                    sb[r] = add_mod(sb[r], acc[0][r], q)
                    sa[r] = add_mod(sa[r], acc[1][r], q)
            acc = (sb, sa)
            if g != 0:
                acc = o.hrot(level, acc, keys[gstr], gstr)
        rb, ra = o.rescale_ct(level, np.stack(acc))
        return (rb, ra), pt_scale * ct_scale / o.rescale_prime_prod(level)
    if bs_set == [0]:
        # Hoist.cu:706-808 (single baby step 0 after the swap)
        mu = o.modup(level, ax)
        bxp = h.pseudo_modup(bx)
        final = None
        for g in gs_set:
            pt = enc[(g, 0)]
            if g == 0:
                final = (h.pmul(h.pseudo_modup(bx), pt), h.pmul(h.pseudo_modup(ax), pt))
        for g in gs_set:
            if g == 0:
                continue
            tb, ta = h.key_mult(mu, keys[g])
            tb = h.add(tb, bxp, rows=h.nq)
            pb, pa = h.permute(h.pmul(tb, enc[(g, 0)]), g), h.permute(h.pmul(ta, enc[(g, 0)]), g)
            final = (pb, pa) if final is None else (h.add(final[0], pb), h.add(final[1], pa))
    else:
        # baby steps: BSFusedKeyMult (Hoist.cu:21-78, 207-327)
        rot = [b for b in bs_set if b]
        bsct = {}
        if rot:
            ob, oa = o.hoisted_rotate(level, (bx, ax), [keys[r] for r in rot], rot)
            for j, r in enumerate(rot):
                bsct[r] = (ob[j], oa[j])
        if 0 in bs_set:
            bsct[0] = (h.pseudo_modup(bx), h.pseudo_modup(ax))
        # giant-step plaintext accumulation: GSFusedKernel (Hoist.cu:81-118)
        acc = {}
        for g in gs_set:
            sb, sa = h.zeros(), h.zeros()
            for b in bs_set:
                if (g, b) not in enc:
                    continue
                sb = h.add(sb, h.pmul(bsct[b][0], enc[(g, b)]))
                sa = h.add(sa, h.pmul(bsct[b][1], enc[(g, b)]))
            acc[g] = (sb, sa)
        final = acc.get(0, (h.zeros(), h.zeros()))
        # EvaluateGiantStepOptimized (Hoist.cu:860-975)
        for g in gs_set:
            if g == 0:
                continue
            md = o.moddown(level, acc[g][1])
            mu = o.modup(level, md)
            tb, ta = h.key_mult(mu, keys[g])
            final = (h.add(final[0], h.permute(tb, g)), h.add(final[1], h.permute(ta, g)))
            final = (h.add(final[0], h.permute(acc[g][0], g)), final[1])
    # EvaluateFinalModDown (Hoist.cu:460-488)
    rb = o.moddown_rescale(level, final[0])
    ra = o.moddown_rescale(level, final[1])
    return (rb, ra), pt_scale * ct_scale / o.rescale_prime_prod(level)


# ---------------------------------------------------------------------------
# Op programs (compiled EvalPoly / EvalMod / Boot): each op restated on the
# oracle's primitives with the semantics of the reference Context
# (src/core/Context.cpp): MultUnsafe Ct x Const / Ct x Ct at a target level
# reading past extra terminal primes, CAccum, Add / Sub with mixed Rx,
# RelinearizeRescale, Rescale, LevelDown, HConj, MultImaginaryUnit,
# ModUpToMax, HRotAdd, linear transforms.
# ---------------------------------------------------------------------------

K_CONST_MULT, K_TENSOR, K_CACCUM, K_ADD_CONST, K_ADD, K_RELIN_RESCALE, K_RESCALE, K_LEVEL_DOWN, \
    K_COPY, K_SET_SCALE, K_SUB, K_HCONJ, K_MULT_IMAG, K_MODUP_TO_MAX, K_HROT_ADD, K_LIN_TRANS, K_SET_SLOTS = range(17)


class Ct:
    def __init__(self, level, parts, scale):
        self.level = level
        self.parts = [np.asarray(p, dtype=np.uint32) for p in parts]
        self.scale = scale


def _ter(o, level):
    return o.level_np(level)[1]


def _qprimes(o, level):
    return [int(p) for p in o.primes(level)]


def _cmul_rows(o, level, x, front, c, cfront):
    qs = _qprimes(o, level)
    out = np.zeros((len(qs), o.n), dtype=np.uint32)
    for r, q in enumerate(qs):
        out[r] = mont_mul(x[front + r], c[cfront + r], q)
    return out


def run_program(o, prog, inp, mult_key=None, conj_key=None, rot_keys=None, lts=None, sse_keys=None,
                min_ks=False):
    """Runs a compiled program (the dict of chd_program_json) on `inp`
    (a Ct); returns the output Ct.  sse_keys = (dts, std) selects
    ModUpToMax with sparse-secret encapsulation."""
    consts = []
    for level, scale, value in prog["consts"]:
        consts.append((level, scale, o.encode_const(level, scale, value)))
    regs = {prog["input"]: inp}

    def acc_part(level, terms, p):
        qs = _qprimes(o, level)
        out = np.zeros((len(qs), o.n), dtype=np.uint32)
        for ct, front, c, cfront in terms:
            if p >= len(ct.parts):
                continue
            for r, q in enumerate(qs):
                v = ct.parts[p][front + r] if c is None else mont_mul(ct.parts[p][front + r], c[cfront + r], q)
                out[r] = add_mod(out[r], v, q)
        return out

    for op in prog["ops"]:
        k, d, a, b, lvl = op["k"], op["d"], op["a"], op["b"], op["l"]
        if k in (K_CONST_MULT, K_LEVEL_DOWN):
            x = regs[a]
            level = x.level if k == K_LEVEL_DOWN else lvl
            cl, cs, cx = consts[op["c"]]
            parts = [_cmul_rows(o, level, p, _ter(o, x.level) - _ter(o, level), cx, _ter(o, cl) - _ter(o, level))
                     for p in x.parts]
            y = Ct(level, parts, x.scale * cs)
            if k == K_LEVEL_DOWN:
                y = Ct(level - 1, o.rescale_ct(level, np.stack(y.parts)), y.scale / o.rescale_prime_prod(level))
            regs[d] = y
        elif k == K_TENSOR:
            x, y = regs[a], regs[b]
            nq = o.num_q(lvl)
            fx, fy = _ter(o, x.level) - _ter(o, lvl), _ter(o, y.level) - _ter(o, lvl)
            d0, d1, d2 = o.tensor(lvl, x.parts[0][fx:fx + nq], x.parts[1][fx:fx + nq],
                                  y.parts[0][fy:fy + nq], y.parts[1][fy:fy + nq])
            regs[d] = Ct(lvl, [d0, d1, d2], x.scale * y.scale)
        elif k == K_CACCUM:
            terms = []
            scale = 0.0
            for s, c in zip(op["s"], op["cs"]):
                x = regs[s]
                cl, cs, cx = consts[c]
                terms.append((x, _ter(o, x.level) - _ter(o, lvl), cx, _ter(o, cl) - _ter(o, lvl)))
                if scale == 0:
                    scale = x.scale * cs
            nparts = 2
            if op["p"] >= 0:
                pl = regs[op["p"]]
                terms.append((pl, 0, None, 0))
                nparts = len(pl.parts)
                if scale == 0:
                    scale = pl.scale
            regs[d] = Ct(lvl, [acc_part(lvl, terms, p) for p in range(nparts)], scale)
        elif k == K_ADD_CONST:
            x = regs[a]
            cl, cs, cx = consts[op["c"]]
            qs = _qprimes(o, x.level)
            f = _ter(o, cl) - _ter(o, x.level)
            bx = np.stack([add_mod(x.parts[0][r], cx[f + r], q) for r, q in enumerate(qs)])
            regs[d] = Ct(x.level, [bx] + list(x.parts[1:]), x.scale)
        elif k in (K_ADD, K_SUB):
            x, y = regs[a], regs[b]
            qs = _qprimes(o, x.level)
            both = min(len(x.parts), len(y.parts))
            parts = []
            for p in range(both):
                if k == K_ADD:
                    parts.append(np.stack([add_mod(x.parts[p][r], y.parts[p][r], q) for r, q in enumerate(qs)]))
                else:
                    parts.append(np.stack([((x.parts[p][r].astype(np.int64) - y.parts[p][r]) % q).astype(np.uint32)
                                           for r, q in enumerate(qs)]))
            if len(x.parts) == 3 and both == 2:
                parts.append(x.parts[2])
            elif len(y.parts) == 3 and both == 2:
                parts.append(y.parts[2])
            regs[d] = Ct(x.level, parts, x.scale)
        elif k == K_RELIN_RESCALE:
            x = regs[a]
            rb, ra = o.relinearize(x.level, x.parts, mult_key, rescale=True)
            regs[d] = Ct(x.level - 1, [rb, ra], x.scale / o.rescale_prime_prod(x.level))
        elif k == K_RESCALE:
            x = regs[a]
            regs[d] = Ct(x.level - 1, list(o.rescale_ct(x.level, np.stack(x.parts))),
                         x.scale / o.rescale_prime_prod(x.level))
        elif k == K_COPY:
            x = regs[a]
            regs[d] = Ct(x.level, [p.copy() for p in x.parts], x.scale)
        elif k == K_SET_SCALE:
            regs[d].scale = op["sc"]
        elif k == K_SET_SLOTS:
            pass  # slot counts only normalise rotation distances, which the program states
        elif k == K_HCONJ:
            x = regs[a]
            rb, ra = o.hconj(x.level, x.parts, conj_key)
            regs[d] = Ct(x.level, [rb, ra], x.scale)
        elif k == K_MULT_IMAG:
            x = regs[a]
            regs[d] = Ct(x.level, [o.mult_imag_unit(x.level, p) for p in x.parts], x.scale)
        elif k == K_MODUP_TO_MAX:
            x = regs[a]
            if sse_keys is not None:
                rb, ra = o.modup_to_max_sse(x.parts[0], x.parts[1], sse_keys[0], sse_keys[1])
            else:
                rb, ra = o.modup_to_max(x.parts[0], x.parts[1])
            regs[d] = Ct(o.max_level, [rb, ra], x.scale)
        elif k == K_HROT_ADD:
            x, y = regs[a], regs[b]
            rb, ra = o.hrot(x.level, x.parts, rot_keys[op["r"]], op["r"])
            qs = _qprimes(o, x.level)
            regs[d] = Ct(x.level, [np.stack([add_mod(rb[r], y.parts[0][r], q) for r, q in enumerate(qs)]),
                                   np.stack([add_mod(ra[r], y.parts[1][r], q) for r, q in enumerate(qs)])], x.scale)
        elif k == K_LIN_TRANS:
            x = regs[a]
            plan = lts[op["r"]]
            (rb, ra), sc = lt_evaluate(o, plan["level"], x.parts, x.scale, plan["pts"], plan["scale"], rot_keys,
                                       min_ks=min_ks)
            regs[d] = Ct(plan["level"] - 1, [rb, ra], sc)
        else:
            raise ValueError(f"unknown op {k}")
    return regs[prog["output"]]


def plain_program(prog, x):
    """Evaluates a program on plain values (constants by their value; scales,
    rescaling and key switching are identities on the message), which is the
    polynomial the compiled program computes (cf. EvalPoly::PlainEvaluate,
    EvalPoly.cpp:845-854)."""
    regs = {prog["input"]: np.asarray(x, dtype=np.float64)}
    vals = [c[2] for c in prog["consts"]]
    for op in prog["ops"]:
        k, d, a, b = op["k"], op["d"], op["a"], op["b"]
        if k == K_CONST_MULT:
            regs[d] = regs[a] * vals[op["c"]]
        elif k == K_TENSOR:
            regs[d] = regs[a] * regs[b]
        elif k == K_CACCUM:
            v = sum(regs[s] * vals[c] for s, c in zip(op["s"], op["cs"]))
            if op["p"] >= 0:
                v = v + regs[op["p"]]
            regs[d] = v
        elif k == K_ADD_CONST:
            regs[d] = regs[a] + vals[op["c"]]
        elif k == K_ADD:
            regs[d] = regs[a] + regs[b]
        elif k == K_SUB:
            regs[d] = regs[a] - regs[b]
        elif k in (K_RELIN_RESCALE, K_RESCALE, K_LEVEL_DOWN, K_COPY):
            regs[d] = regs[a]
        elif k in (K_SET_SCALE, K_SET_SLOTS):
            pass
        else:
            raise ValueError(f"plain evaluation does not cover op {k}")
    return regs[prog["output"]]


# ---------------------------------------------------------------------------
# Test-only key generation for sparse-secret encapsulation (the reference's
# UserInterface::PrepareBasicEvks, UserInterface.cu:342-356 with PrepareEvk,
# :366-458): b = e - a s_enc + P s_target on the q primes of the digit, a
# uniform, e a rounded Gaussian (sigma 3.2) in the evaluation domain.
# ---------------------------------------------------------------------------

def _error_row(o, g, e):
    q = int(o.all_primes()[g])
    limb = np.where(e < 0, q + e, e).astype(np.uint32)
    return o.ntt_limb(g, limb, mont=True)


def gen_evk_rows(o, seed, gidx, nq, enc_s, tgt_s, p_mont):
    """One-digit key over the rows `gidx` (q rows first): target term on the
    first nq rows with the Montgomery constants p_mont[r]."""
    rng = np.random.default_rng(seed)
    primes = o.all_primes()
    kb = np.zeros((1, len(gidx), o.n), dtype=np.uint32)
    ka = np.zeros_like(kb)
    e = np.rint(rng.normal(0, 3.2, o.n)).astype(np.int64)
    for r, g in enumerate(gidx):
        q = int(primes[g])
        a = rng.integers(0, q, o.n, dtype=np.int64).astype(np.uint32)
        b = _error_row(o, g, e)
        b = ((b.astype(np.int64) - mont_mul(a, enc_s[g], q)) % q).astype(np.uint32)
        if r < nq:
            b = add_mod(b, mont_mul(tgt_s[g], p_mont[r], q), q)
        kb[0, r] = b
        ka[0, r] = a
    return kb, ka


def gen_sse_keys(o, seed, dense_s, sparse_s):
    """(dense-to-sparse key over [num_q(-1) + sse aux], sparse-to-dense key
    over [L + alpha] as one digit)."""
    primes = [int(p) for p in o.all_primes()]
    m, t = o.level_np(-1)
    nb = m + t
    L, alpha = o.L, o.alpha
    g_dts = list(range(o.max_ter - t, o.max_ter + m)) + [L + j for j in range(nb)]
    p_dts = []
    for g in g_dts[:nb]:
        v = 1
        for j in range(nb):
            v = v * primes[L + j] % primes[g]
        p_dts.append(v * 2 ** 32 % primes[g])
    dts = gen_evk_rows(o, seed, g_dts, nb, sparse_s, dense_s, p_dts)
    g_std = list(range(L + alpha))
    p_std = []
    for g in g_std[:L]:
        v = 1
        for j in range(alpha):
            v = v * primes[L + j] % primes[g]
        p_std.append(v * 2 ** 32 % primes[g])
    std = gen_evk_rows(o, seed + 1, g_std, L, dense_s, sparse_s, p_std)
    return dts, std
