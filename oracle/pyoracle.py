"""ctypes binding of the CPU oracle (oracle/oracle.c) — test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It never stands in for the CUDA path.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build():
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        sig = {
            "orc_create": (vp, [C.c_int, C.c_double, C.c_int, i32p, C.c_int, u32p,
                                C.c_int, u32p, C.c_int, C.c_void_p, C.c_int,
                                C.c_int, C.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_last_error": (C.c_char_p, []),
            "orc_degree": (C.c_int, [vp]),
            "orc_max_level": (C.c_int, [vp]),
            "orc_alpha": (C.c_int, [vp]),
            "orc_L": (C.c_int, [vp]),
            "orc_max_ter": (C.c_int, [vp]),
            "orc_level_np": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "orc_beta": (C.c_int, [vp, C.c_int]),
            "orc_prime_vector": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, u32p]),
            "orc_prime_gidx": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, i32p]),
            "orc_scale": (C.c_double, [vp, C.c_int]),
            "orc_rescale_prime_prod": (C.c_double, [vp, C.c_int]),
            "orc_galois_factor": (C.c_int, [vp, C.c_int]),
            "orc_twiddles": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "orc_ntt": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, u32p, C.c_int]),
            "orc_intt": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, u32p, C.c_int]),
            "orc_ntt_limb": (C.c_int, [vp, C.c_int, u32p, C.c_int]),
            "orc_intt_limb": (C.c_int, [vp, C.c_int, u32p, C.c_int]),
            "orc_bconv": (C.c_int, [vp, i32p, C.c_int, i32p, u32p, C.c_int, u32p]),
            "orc_bconv_ref_schedule": (C.c_int, [vp, i32p, C.c_int, i32p, u32p, C.c_int, u32p]),
            "orc_bconv_table": (C.c_int, [u32p, C.c_int, u32p, C.c_int, i32p]),
            "orc_modup": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "orc_moddown": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "orc_rescale": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "orc_moddown_rescale": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "orc_tensor": (C.c_int, [vp, C.c_int, C.c_int, u32p, u32p, u32p, u32p, u32p, u32p, u32p]),
            "orc_permute": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, u32p, u32p]),
            "orc_mult_imag_unit": (C.c_int, [vp, C.c_int, C.c_int, u32p, u32p]),
            "orc_hmult": (C.c_int, [vp, C.c_int, u32p, u32p, u32p, u32p, u32p, u32p,
                                    C.c_int, u32p, u32p]),
            "orc_mult_key": (C.c_int, [vp, C.c_int, u32p, u32p, u32p, u32p, u32p, u32p]),
            "orc_hrot": (C.c_int, [vp, C.c_int, u32p, u32p, u32p, u32p, C.c_int, u32p, u32p]),
            "orc_hconj": (C.c_int, [vp, C.c_int, u32p, u32p, u32p, u32p, u32p, u32p]),
            "orc_rescale_ct": (C.c_int, [vp, C.c_int, C.c_int, u32p, u32p]),
            "orc_hoisted_rotate": (C.c_int, [vp, C.c_int, u32p, u32p, C.c_int, i32p,
                                             C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                             u32p, u32p]),
            "orc_gen_secret": (C.c_int, [vp, C.c_uint64, C.c_int, u32p]),
            "orc_gen_evk": (C.c_int, [vp, C.c_uint64, u32p, u32p, u32p, u32p]),
            "orc_gen_mult_key": (C.c_int, [vp, C.c_uint64, u32p, u32p, u32p]),
            "orc_gen_rot_key": (C.c_int, [vp, C.c_uint64, u32p, C.c_int, u32p, u32p]),
            "orc_gen_conj_key": (C.c_int, [vp, C.c_uint64, u32p, u32p, u32p]),
            "orc_encrypt": (C.c_int, [vp, C.c_uint64, u32p, C.c_int, u32p, u32p, u32p]),
            "orc_decrypt": (C.c_int, [vp, u32p, C.c_int, u32p, u32p, u32p]),
            "orc_encode": (C.c_int, [vp, C.c_int, C.c_double, f64p, f64p, C.c_int, C.c_int, u32p]),
            "orc_decode": (C.c_int, [vp, C.c_int, C.c_double, u32p, C.c_int, f64p, f64p]),
            "orc_encode_const": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_int, u32p]),
            "orc_modup_to_max": (C.c_int, [vp, u32p, u32p, u32p, u32p]),
            "orc_modup_to_max_sse": (C.c_int, [vp, u32p, u32p, u32p, u32p, u32p, u32p, u32p, u32p]),
            "orc_relinearize": (C.c_int, [vp, C.c_int, u32p, u32p, u32p, u32p, u32p, C.c_int, u32p, u32p]),
            "orc_uniform": (C.c_int, [vp, C.c_uint64, C.c_int, C.c_int, C.c_int, u32p]),
            "orc_mont_reduce_lazy": (C.c_int32, [C.c_int64, C.c_uint32, C.c_int32]),
            "orc_mont_mult_lazy": (C.c_int32, [C.c_int32, C.c_int32, C.c_uint32, C.c_int32]),
            "orc_mont_reduce": (C.c_uint32, [C.c_int64, C.c_uint32, C.c_int32]),
            "orc_mont_mult": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32]),
            "orc_normalize": (C.c_int32, [C.c_uint32, C.c_uint32]),
            "orc_pow_mod": (C.c_uint32, [C.c_uint32, C.c_int64, C.c_uint32]),
            "orc_inv_mod": (C.c_uint32, [C.c_uint32, C.c_uint32]),
            "orc_find_generator": (C.c_uint32, [C.c_uint32]),
            "orc_primitive_root": (C.c_uint32, [C.c_int, C.c_uint32]),
            "orc_inv_mod_base": (C.c_int32, [C.c_uint32]),
            "orc_to_mont": (C.c_uint32, [C.c_uint32, C.c_uint32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def load_param_json(path):
    with open(path) as f:
        return json.load(f)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed: {lib().orc_last_error().decode()}")


class Oracle:
    """CPU restatement of the reference evaluator on one parameter set."""

    def __init__(self, params, log_degree=None):
        p = dict(params)
        L = lib()
        self.log_n = int(log_degree if log_degree is not None else p["log_degree"])
        self.n = 1 << self.log_n
        self.params = p
        main = np.asarray(p["main_primes"], dtype=np.uint32)
        aux = np.asarray(p["auxiliary_primes"], dtype=np.uint32)
        ter = np.asarray(p.get("terminal_primes", []), dtype=np.uint32)
        lvl = np.asarray(p["level_config"], dtype=np.int32).reshape(-1)
        add = p.get("additional_base", [0, 0])
        scale = float(1 << int(p["log_default_scale"]))
        self.ptr = L.orc_create(self.log_n, scale, int(p["default_encryption_level"]),
                                lvl, len(p["level_config"]), main, len(main), aux, len(aux),
                                ter.ctypes.data if len(ter) else None, len(ter),
                                int(add[0]), int(add[1]))
        if not self.ptr:
            raise ValueError(L.orc_last_error().decode())
        self.max_level = L.orc_max_level(self.ptr)
        self.alpha = L.orc_alpha(self.ptr)
        self.L = L.orc_L(self.ptr)
        self.max_ter = L.orc_max_ter(self.ptr)
        self.nprimes = self.L + self.alpha
        self.beta_max = -(-self.L // self.alpha)

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_destroy(self.ptr)
            self.ptr = None

    # ---- level model ----
    def level_np(self, level):
        m, t = C.c_int(), C.c_int()
        _check(lib().orc_level_np(self.ptr, level, C.byref(m), C.byref(t)), "level_np")
        return m.value, t.value

    def num_q(self, level):
        m, t = self.level_np(level)
        return m + t

    def beta(self, level):
        return lib().orc_beta(self.ptr, level)

    def primes(self, level, num_aux=0):
        m, t = self.level_np(level)
        out = np.zeros(m + t + num_aux, dtype=np.uint32)
        lib().orc_prime_vector(self.ptr, m, t, num_aux, out)
        return out

    def gidx(self, level, num_aux=0):
        m, t = self.level_np(level)
        out = np.zeros(m + t + num_aux, dtype=np.int32)
        lib().orc_prime_gidx(self.ptr, m, t, num_aux, out)
        return out

    def all_primes(self):
        m, t = self.level_np(self.max_level)
        out = np.zeros(self.nprimes, dtype=np.uint32)
        lib().orc_prime_vector(self.ptr, m, t, self.alpha, out)
        return out

    def scale(self, level):
        return lib().orc_scale(self.ptr, level)

    def rescale_prime_prod(self, level):
        return lib().orc_rescale_prime_prod(self.ptr, level)

    def twiddles(self, gidx):
        tw = np.zeros(self.n, dtype=np.uint32)
        itw = np.zeros(self.n, dtype=np.uint32)
        _check(lib().orc_twiddles(self.ptr, gidx, tw, itw), "twiddles")
        return tw, itw

    # ---- transforms ----
    def ntt(self, level, data, num_aux=0, mont=False):
        m, t = self.level_np(level)
        d = np.ascontiguousarray(data, dtype=np.uint32).copy()
        lib().orc_ntt(self.ptr, m, t, num_aux, d, int(mont))
        return d

    def intt(self, level, data, num_aux=0, mont=True):
        m, t = self.level_np(level)
        d = np.ascontiguousarray(data, dtype=np.uint32).copy()
        lib().orc_intt(self.ptr, m, t, num_aux, d, int(mont))
        return d

    def ntt_limb(self, gidx, limb, mont=False):
        d = np.ascontiguousarray(limb, dtype=np.uint32).copy()
        _check(lib().orc_ntt_limb(self.ptr, gidx, d, int(mont)), "ntt_limb")
        return d

    def intt_limb(self, gidx, limb, mont=True):
        d = np.ascontiguousarray(limb, dtype=np.uint32).copy()
        _check(lib().orc_intt_limb(self.ptr, gidx, d, int(mont)), "intt_limb")
        return d

    # ---- base conversion ----
    @staticmethod
    def bconv_table(src_primes, dst_primes):
        s = np.ascontiguousarray(src_primes, dtype=np.uint32)
        d = np.ascontiguousarray(dst_primes, dtype=np.uint32)
        t = np.zeros(len(d) * len(s), dtype=np.int32)
        lib().orc_bconv_table(s, len(s), d, len(d), t)
        return t

    def bconv(self, xt, table, dst_primes, ref_schedule=False):
        xt = np.ascontiguousarray(xt, dtype=np.int32)
        K = xt.shape[0]
        d = np.ascontiguousarray(dst_primes, dtype=np.uint32)
        out = np.zeros((len(d), self.n), dtype=np.uint32)
        f = lib().orc_bconv_ref_schedule if ref_schedule else lib().orc_bconv
        f(self.ptr, xt, K, np.ascontiguousarray(table, dtype=np.int32), d, len(d), out)
        return out

    # ---- mod switch ----
    def modup(self, level, src):
        nq = self.num_q(level)
        beta = self.beta(level)
        out = np.zeros((beta, nq + self.alpha, self.n), dtype=np.uint32)
        _check(lib().orc_modup(self.ptr, level, np.ascontiguousarray(src, dtype=np.uint32), out), "modup")
        return out

    def moddown(self, level, src):
        out = np.zeros((self.num_q(level), self.n), dtype=np.uint32)
        _check(lib().orc_moddown(self.ptr, level, np.ascontiguousarray(src, dtype=np.uint32), out), "moddown")
        return out

    def rescale(self, level, src):
        out = np.zeros((self.num_q(level - 1), self.n), dtype=np.uint32)
        _check(lib().orc_rescale(self.ptr, level, np.ascontiguousarray(src, dtype=np.uint32), out), "rescale")
        return out

    def moddown_rescale(self, level, src):
        out = np.zeros((self.num_q(level - 1), self.n), dtype=np.uint32)
        _check(lib().orc_moddown_rescale(self.ptr, level, np.ascontiguousarray(src, dtype=np.uint32), out),
               "moddown_rescale")
        return out

    # ---- element-wise ----
    def tensor(self, level, b1, a1, b2, a2):
        m, t = self.level_np(level)
        shp = (m + t, self.n)
        d0, d1, d2 = (np.zeros(shp, dtype=np.uint32) for _ in range(3))
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        lib().orc_tensor(self.ptr, m, t, c(b1), c(a1), c(b2), c(a2), d0, d1, d2)
        return d0, d1, d2

    def permute(self, level, amount, src, num_aux=0):
        m, t = self.level_np(level)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        out = np.zeros_like(s)
        _check(lib().orc_permute(self.ptr, m, t, num_aux, amount, s, out), "permute")
        return out

    def mult_imag_unit(self, level, src):
        m, t = self.level_np(level)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        out = np.zeros_like(s)
        lib().orc_mult_imag_unit(self.ptr, m, t, s, out)
        return out

    # ---- evaluator ----
    def hmult(self, level, a, b, key, rescale=True):
        nq_out = self.num_q(level - 1 if rescale else level)
        ob = np.zeros((nq_out, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_hmult(self.ptr, level, c(a[0]), c(a[1]), c(b[0]), c(b[1]),
                               c(key[0]), c(key[1]), int(rescale), ob, oa), "hmult")
        return ob, oa

    def relinearize(self, level, d, key, rescale=True):
        """Context::Relinearize(Rescale) of three parts d = (d0, d1, d2)."""
        nq = self.num_q(level - 1 if rescale else level)
        ob = np.zeros((nq, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_relinearize(self.ptr, level, c(d[0]), c(d[1]), c(d[2]), c(key[0]), c(key[1]),
                                     int(rescale), ob, oa), "relinearize")
        return ob, oa

    def mult_key(self, level, a, key):
        nq = self.num_q(level)
        ob = np.zeros((nq, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_mult_key(self.ptr, level, c(a[0]), c(a[1]), c(key[0]), c(key[1]), ob, oa),
               "mult_key")
        return ob, oa

    def hrot(self, level, a, key, amount):
        nq = self.num_q(level)
        ob = np.zeros((nq, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_hrot(self.ptr, level, c(a[0]), c(a[1]), c(key[0]), c(key[1]), amount, ob, oa),
               "hrot")
        return ob, oa

    def hconj(self, level, a, key):
        nq = self.num_q(level)
        ob = np.zeros((nq, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_hconj(self.ptr, level, c(a[0]), c(a[1]), c(key[0]), c(key[1]), ob, oa), "hconj")
        return ob, oa

    def rescale_ct(self, level, parts):
        parts = np.ascontiguousarray(parts, dtype=np.uint32)
        out = np.zeros((parts.shape[0], self.num_q(level - 1), self.n), dtype=np.uint32)
        _check(lib().orc_rescale_ct(self.ptr, level, parts.shape[0], parts, out), "rescale_ct")
        return out

    def hoisted_rotate(self, level, a, keys, amounts):
        R = len(amounts)
        tot = self.num_q(level) + self.alpha
        ob = np.zeros((R, tot, self.n), dtype=np.uint32)
        oa = np.zeros_like(ob)
        kb = [np.ascontiguousarray(k[0], dtype=np.uint32) for k in keys]
        ka = [np.ascontiguousarray(k[1], dtype=np.uint32) for k in keys]
        pb = (C.c_void_p * R)(*[k.ctypes.data for k in kb])
        pa = (C.c_void_p * R)(*[k.ctypes.data for k in ka])
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_hoisted_rotate(self.ptr, level, c(a[0]), c(a[1]), R,
                                        np.asarray(amounts, dtype=np.int32), pb, pa, ob, oa),
               "hoisted_rotate")
        return ob, oa

    # ---- client (test-only) ----
    def gen_secret(self, seed, h):
        s = np.zeros((self.nprimes, self.n), dtype=np.uint32)
        _check(lib().orc_gen_secret(self.ptr, seed, h, s), "gen_secret")
        return s

    def _key_buf(self):
        shp = (self.beta_max, self.nprimes, self.n)
        return np.zeros(shp, dtype=np.uint32), np.zeros(shp, dtype=np.uint32)

    def gen_mult_key(self, seed, s):
        kb, ka = self._key_buf()
        _check(lib().orc_gen_mult_key(self.ptr, seed, s, kb, ka), "gen_mult_key")
        return kb, ka

    def gen_rot_key(self, seed, s, amount):
        kb, ka = self._key_buf()
        _check(lib().orc_gen_rot_key(self.ptr, seed, s, amount, kb, ka), "gen_rot_key")
        return kb, ka

    def gen_conj_key(self, seed, s):
        kb, ka = self._key_buf()
        _check(lib().orc_gen_conj_key(self.ptr, seed, s, kb, ka), "gen_conj_key")
        return kb, ka

    def encrypt(self, seed, s, level, pt):
        nq = self.num_q(level)
        bx = np.zeros((nq, self.n), dtype=np.uint32)
        ax = np.zeros_like(bx)
        _check(lib().orc_encrypt(self.ptr, seed, s, level, np.ascontiguousarray(pt, dtype=np.uint32), bx, ax),
               "encrypt")
        return bx, ax

    def decrypt(self, s, level, ct):
        nq = self.num_q(level)
        pt = np.zeros((nq, self.n), dtype=np.uint32)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_decrypt(self.ptr, s, level, c(ct[0]), c(ct[1]), pt), "decrypt")
        return pt

    def encode(self, level, scale, msg, num_aux=0):
        msg = np.asarray(msg, dtype=np.complex128)
        nq = self.num_q(level)
        pt = np.zeros((nq + num_aux, self.n), dtype=np.uint32)
        _check(lib().orc_encode(self.ptr, level, scale, np.ascontiguousarray(msg.real),
                                np.ascontiguousarray(msg.imag), len(msg), num_aux, pt), "encode")
        return pt

    def decode(self, level, scale, pt, num_slots):
        re = np.zeros(num_slots)
        im = np.zeros(num_slots)
        _check(lib().orc_decode(self.ptr, level, scale, np.ascontiguousarray(pt, dtype=np.uint32),
                                num_slots, re, im), "decode")
        return re + 1j * im

    def encode_const(self, level, scale, value, num_aux=0):
        out = np.zeros(self.num_q(level) + num_aux, dtype=np.uint32)
        lib().orc_encode_const(self.ptr, level, scale, value, num_aux, out)
        return out

    def modup_to_max(self, bx, ax):
        """BootContext::ModUpToMax without sparse-secret encapsulation
        (BootContext.cpp:186-270): level -1 (bx, ax) -> top level."""
        nq = self.num_q(self.max_level)
        rb = np.zeros((nq, self.n), dtype=np.uint32)
        ra = np.zeros((nq, self.n), dtype=np.uint32)
        _check(lib().orc_modup_to_max(self.ptr, np.ascontiguousarray(bx, dtype=np.uint32),
                                      np.ascontiguousarray(ax, dtype=np.uint32), rb, ra), "modup_to_max")
        return rb, ra

    def modup_to_max_sse(self, bx, ax, dts, std):
        """ModUpToMax with sparse-secret encapsulation (BootContext.cpp:
        186-270); dts = (kb, ka) [1][num_q(-1) + sse aux][N], std = (kb, ka)
        with digit 0 over [L + alpha][N]."""
        nq = self.num_q(self.max_level)
        rb = np.zeros((nq, self.n), dtype=np.uint32)
        ra = np.zeros((nq, self.n), dtype=np.uint32)
        c = lambda x: np.ascontiguousarray(x, dtype=np.uint32)
        _check(lib().orc_modup_to_max_sse(self.ptr, c(bx), c(ax), c(dts[0]), c(dts[1]), c(std[0][0]), c(std[1][0]),
                                          rb, ra), "modup_to_max_sse")
        return rb, ra

    def uniform(self, seed, level, num_aux=0):
        m, t = self.level_np(level)
        out = np.zeros((m + t + num_aux, self.n), dtype=np.uint32)
        lib().orc_uniform(self.ptr, seed, m, t, num_aux, out)
        return out
