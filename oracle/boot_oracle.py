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


def lt_evaluate(o, level, ct, ct_scale, pts, pt_scale, keys):
    """HoistHandler::Evaluate for the compiled map `pts` = [(gs, bs, msg)];
    keys = {rotation: (kb, ka)}.  Returns ((bx, ax) at level - 1, scale)."""
    h = HoistOracle(o, level)
    bx, ax = ct
    enc = {(g, b): o.encode(level, pt_scale, m, num_aux=h.alpha) for g, b, m in pts}
    bs_set = sorted({b for _, b, _ in pts})
    gs_set = sorted({g for g, _, _ in pts})
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
