"""ctypes binding of oracle/_ref/libcheddar_ref.so: the reference's own
evaluator library (scale-snu/cheddar-fhe src/core, src/extension,
src/UserInterface.cu) compiled for sm_100a by `make -C oracle ref`, driven
through oracle/ref_pin/ref_driver.cu.

Test infrastructure only (tests/ and bench.py's reference legs): it runs the
reference on the GPU so that parity tests can compare this library's
residues with the reference's on identical inputs and keys, and so that the
bench can time the reference beside this library.  The reference generates
its secret from std::random_device (include/Random.h:78-79): keys and fresh
encryptions differ per process, so every comparison exports them from here
and imports them into the library under test and the CPU oracle.

The reference exits the process on a failed assertion
(include/common/Assert.h:9-21); the wrappers here only pass valid inputs.
"""
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcheddar_ref.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, ip, dp, u32p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p
        sig = {
            "refx_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, u32p, C.c_int, u32p, C.c_int,
                                      u32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p)]),
            "refx_destroy": (None, [vp]),
            "refx_max_level": (C.c_int, [vp]),
            "refx_alpha": (C.c_int, [vp]),
            "refx_dnum": (C.c_int, [vp]),
            "refx_level_np": (None, [vp, C.c_int, C.c_int, ip, ip]),
            "refx_test_scale": (C.c_double, [vp, C.c_int]),
            "refx_scale": (C.c_double, [vp, C.c_int]),
            "refx_prime_vector": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, u32p]),
            "refx_key_index_mult": (C.c_int, []),
            "refx_key_index_conj": (C.c_int, []),
            "refx_key_index_dts": (C.c_int, []),
            "refx_key_index_std": (C.c_int, []),
            "refx_prepare_rotation": (C.c_int, [vp, C.c_int]),
            "refx_key_shape": (C.c_int, [vp, C.c_int, ip, ip, ip, ip]),
            "refx_key_export": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "refx_ct_new": (C.c_void_p, []),
            "refx_ct_free": (None, [vp]),
            "refx_ct_info": (None, [vp, ip, ip, ip, ip, dp, ip]),
            "refx_ct_export": (C.c_int, [vp, vp, u32p, u32p, u32p]),
            "refx_ct_import": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, u32p, u32p]),
            "refx_ct_encrypt": (C.c_int, [vp, vp, C.c_int, C.c_void_p, C.c_void_p, C.c_int]),
            "refx_decrypt_decode": (C.c_int, [vp, vp, C.c_void_p, C.c_void_p]),
            "refx_decrypt": (C.c_int, [vp, vp, u32p, C.POINTER(C.c_double), ip]),
            "refx_decode": (C.c_int, [vp, C.c_int, C.c_double, C.c_int, u32p, C.c_void_p, C.c_void_p]),
            "refx_encode": (C.c_int, [vp, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_int, u32p]),
            "refx_hmult": (C.c_int, [vp, vp, vp, vp, C.c_int]),
            "refx_hrot": (C.c_int, [vp, vp, vp, C.c_int]),
            "refx_hconj": (C.c_int, [vp, vp, vp]),
            "refx_rescale": (C.c_int, [vp, vp, vp]),
            "refx_unary": (C.c_int, [vp, C.c_char_p, vp, vp, C.c_int]),
            "refx_binary": (C.c_int, [vp, C.c_char_p, vp, vp, vp, C.c_int]),
            "refx_ntt": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, u32p, C.c_int, C.c_int, C.c_int]),
            "refx_modup": (C.c_int, [vp, C.c_int, u32p, u32p]),
            "refx_moddown": (C.c_int, [vp, C.c_int, C.c_int, u32p, u32p]),
            "refx_hoisted_baby_steps": (C.c_int, [vp, vp, C.c_void_p, C.c_int, C.c_void_p]),
            "refx_boot_prepare": (C.c_int, [vp, C.c_int, C.c_void_p, C.c_int, ip]),
            "refx_boot": (C.c_int, [vp, vp, vp, C.c_int]),
            "refx_time_hmult": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]),
            "refx_time_hmult_set": (C.c_int, [vp, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.POINTER(C.c_float)]),
            "refx_time_hrot": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]),
            "refx_time_ntt_roundtrip": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]),
            "refx_time_boot": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]),
            "refx64_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, vp, C.c_int, vp, C.c_int,
                                        vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
            "refx64_destroy": (None, [vp]),
            "refx64_ntt": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int]),
            "refx64_modup": (C.c_int, [vp, C.c_int, vp, vp]),
            "refx64_moddown": (C.c_int, [vp, C.c_int, C.c_int, vp, vp]),
            "refx64_hmult": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, C.c_int, vp, vp, C.c_int, vp, vp]),
            "refx64_hrot": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, vp, vp, C.c_int, vp, vp]),
            "refx64_hconj": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, vp, vp, vp, vp]),
            "refx64_op": (C.c_int, [vp, C.c_char_p, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, C.c_int,
                                    C.c_double, C.c_double, vp, vp, vp, vp]),
            "refx64_time_hmult": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(C.c_float)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} failed: {rc}")


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class RefContext:
    """The reference's Context / BootContext with its test client
    (UserInterface): secret, mult / conj / sparse-secret keys."""

    def __init__(self, params):
        p = json.loads(params) if isinstance(params, str) else params
        self.params = p
        L = lib()
        lv = np.array([x for pair in p["level_config"] for x in pair], dtype=np.int32)
        main = _u32(p["main_primes"])
        aux = _u32(p["auxiliary_primes"])
        ter = _u32(p.get("terminal_primes", []) or [0])
        n_ter = len(p.get("terminal_primes", []))
        add = p.get("additional_base", [0, 0])
        self._keep = (lv, main, aux, ter)
        self.ptr = C.c_void_p()
        _chk(L.refx_create(p["log_degree"], p["log_default_scale"], p["default_encryption_level"],
                           len(p["level_config"]), lv.ctypes.data, main.ctypes.data, len(main), aux.ctypes.data,
                           len(aux), ter.ctypes.data, n_ter, add[0], add[1], p.get("dense_hamming_weight", 0),
                           p.get("sparse_hamming_weight", 0), int(bool(p.get("boot", False))),
                           p.get("num_cts_levels", 0), p.get("num_stc_levels", 0), C.byref(self.ptr)), "create")
        self.n = 1 << p["log_degree"]
        self.max_level = L.refx_max_level(self.ptr)
        self.alpha = L.refx_alpha(self.ptr)
        self.dnum = L.refx_dnum(self.ptr)

    def close(self):
        if getattr(self, "ptr", None) is not None and self.ptr.value:
            lib().refx_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def level_np(self, level, num_aux=0):
        m, t = C.c_int(), C.c_int()
        lib().refx_level_np(self.ptr, level, num_aux, C.byref(m), C.byref(t))
        return m.value, t.value

    def test_scale(self, level):
        return lib().refx_test_scale(self.ptr, level)

    def scale(self, level):
        return lib().refx_scale(self.ptr, level)

    def prime_vector(self, num_main, num_ter, num_aux):
        out = np.zeros(num_main + num_ter + num_aux, dtype=np.uint32)
        k = lib().refx_prime_vector(self.ptr, num_main, num_ter, num_aux, out.ctypes.data)
        return out[:k]

    # ---- keys ----
    MULT = property(lambda self: lib().refx_key_index_mult())
    CONJ = property(lambda self: lib().refx_key_index_conj())
    DTS = property(lambda self: lib().refx_key_index_dts())
    STD = property(lambda self: lib().refx_key_index_std())

    def prepare_rotation(self, r):
        _chk(lib().refx_prepare_rotation(self.ptr, r), "PrepareRotationKey")

    def key_shape(self, idx):
        b, m, t, a = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        if lib().refx_key_shape(self.ptr, idx, C.byref(b), C.byref(m), C.byref(t), C.byref(a)) != 0:
            raise KeyError(idx)
        return b.value, m.value, t.value, a.value

    def key(self, idx):
        """(bx, ax) as [beta][np][N] uint32, and the key basis (main, ter, aux)."""
        beta, m, t, a = self.key_shape(idx)
        bx = np.zeros((beta, m + t + a, self.n), dtype=np.uint32)
        ax = np.zeros_like(bx)
        _chk(lib().refx_key_export(self.ptr, idx, bx.ctypes.data, ax.ctypes.data), "key export")
        return bx, ax, (m, t, a)

    # ---- ciphertexts ----
    def ct(self):
        return RefCiphertext(self)

    def encrypt(self, level, msg):
        msg = np.asarray(msg, dtype=np.complex128)
        re = np.ascontiguousarray(msg.real)
        im = np.ascontiguousarray(msg.imag)
        c = RefCiphertext(self)
        _chk(lib().refx_ct_encrypt(self.ptr, c.ptr, level, re.ctypes.data, im.ctypes.data, len(msg)), "encrypt")
        return c

    def import_ct(self, num_main, num_ter, num_aux, parts, scale, num_slots):
        c = RefCiphertext(self)
        bx, ax = _u32(parts[0]), _u32(parts[1])
        _chk(lib().refx_ct_import(self.ptr, c.ptr, num_main, num_ter, num_aux, scale, num_slots, bx.ctypes.data,
                                  ax.ctypes.data), "ct import")
        return c

    def decrypt_decode(self, c):
        ns = c.info()["num_slots"]
        re = np.zeros(ns)
        im = np.zeros(ns)
        _chk(lib().refx_decrypt_decode(self.ptr, c.ptr, re.ctypes.data, im.ctypes.data), "decrypt")
        return re + 1j * im

    def decrypt(self, c):
        """(plaintext residues [num_q][N], scale, num_slots) of a ciphertext."""
        inf = c.info()
        out = np.zeros((inf["num_main"] + inf["num_ter"], self.n), dtype=np.uint32)
        sc, ns = C.c_double(), C.c_int()
        _chk(lib().refx_decrypt(self.ptr, c.ptr, out.ctypes.data, C.byref(sc), C.byref(ns)), "decrypt")
        return out, sc.value, ns.value

    def decode(self, level, scale, num_slots, pt):
        p = _u32(pt)
        re = np.zeros(num_slots)
        im = np.zeros(num_slots)
        _chk(lib().refx_decode(self.ptr, level, scale, num_slots, p.ctypes.data, re.ctypes.data, im.ctypes.data),
             "decode")
        return re + 1j * im

    def encode(self, level, scale, msg, num_aux=0):
        msg = np.asarray(msg, dtype=np.complex128)
        re = np.ascontiguousarray(msg.real)
        im = np.ascontiguousarray(msg.imag)
        m, t = self.level_np(level)
        out = np.zeros((m + t + num_aux, self.n), dtype=np.uint32)
        _chk(lib().refx_encode(self.ptr, level, scale, re.ctypes.data, im.ctypes.data, len(msg), num_aux,
                               out.ctypes.data), "encode")
        return out

    # ---- evaluator ----
    def HMult(self, a, b, rescale=True):
        r = RefCiphertext(self)
        _chk(lib().refx_hmult(self.ptr, r.ptr, a.ptr, b.ptr, int(rescale)), "HMult")
        return r

    def HRot(self, a, rot):
        r = RefCiphertext(self)
        _chk(lib().refx_hrot(self.ptr, r.ptr, a.ptr, rot), "HRot")
        return r

    def HConj(self, a):
        r = RefCiphertext(self)
        _chk(lib().refx_hconj(self.ptr, r.ptr, a.ptr), "HConj")
        return r

    def Rescale(self, a):
        r = RefCiphertext(self)
        _chk(lib().refx_rescale(self.ptr, r.ptr, a.ptr), "Rescale")
        return r

    def unary(self, op, a, arg=0):
        r = RefCiphertext(self)
        _chk(lib().refx_unary(self.ptr, op.encode(), r.ptr, a.ptr, arg), op)
        return r

    def binary(self, op, a, b, arg=0):
        r = RefCiphertext(self)
        _chk(lib().refx_binary(self.ptr, op.encode(), r.ptr, a.ptr, b.ptr, arg), op)
        return r

    def ntt(self, num_main, num_ter, num_aux, data, inverse=False, montgomery=False):
        d = _u32(data).copy()
        count = d.size // ((num_main + num_ter + num_aux) * self.n)
        _chk(lib().refx_ntt(self.ptr, num_main, num_ter, num_aux, d.ctypes.data, count, int(inverse),
                            int(montgomery)), "NTT")
        return d

    def modup(self, level, src):
        m, t = self.level_np(level)
        q = m + t
        max_ter = len(self.params.get("terminal_primes", []))
        beta = -(-(q + max_ter - t) // self.alpha)
        out = np.zeros((beta, q + self.alpha, self.n), dtype=np.uint32)
        s = _u32(src)
        _chk(lib().refx_modup(self.ptr, level, s.ctypes.data, out.ctypes.data), "ModUp")
        return out

    def moddown(self, level, kind, src):
        """kind 0 ModDown, 1 Rescale, 2 ModDownAndRescale."""
        m, t = self.level_np(level if kind == 0 else level - 1)
        out = np.zeros((m + t, self.n), dtype=np.uint32)
        s = _u32(src)
        _chk(lib().refx_moddown(self.ptr, level, kind, s.ctypes.data, out.ctypes.data), "ModDown")
        return out

    def hoisted_baby_steps(self, c, rots):
        outs = [RefCiphertext(self) for _ in rots]
        r = np.array(rots, dtype=np.int32)
        arr = (C.c_void_p * len(rots))(*[o.ptr.value for o in outs])
        _chk(lib().refx_hoisted_baby_steps(self.ptr, c.ptr, r.ctypes.data, len(rots), arr), "hoisted baby steps")
        return outs

    # ---- bootstrapping ----
    def boot_prepare(self, num_slots):
        cap = 4096
        out = np.zeros(cap, dtype=np.int32)
        n = C.c_int()
        _chk(lib().refx_boot_prepare(self.ptr, num_slots, out.ctypes.data, cap, C.byref(n)), "boot prepare")
        return [int(x) for x in out[:n.value]]

    def Boot(self, c, min_ks=False):
        r = RefCiphertext(self)
        _chk(lib().refx_boot(self.ptr, r.ptr, c.ptr, int(min_ks)), "Boot")
        return r

    # ---- device timing (total ms over `iters` calls) ----
    def time_hmult(self, a, b, iters, warmup=3, rescale=True):
        ms = C.c_float()
        _chk(lib().refx_time_hmult(self.ptr, a.ptr, b.ptr, int(rescale), warmup, iters, C.byref(ms)), "time HMult")
        return ms.value

    def time_hmult_set(self, a_list, b_list, iters, warmup=3, rescale=True):
        n = len(a_list)
        pa = (C.c_void_p * n)(*[c.ptr.value for c in a_list])
        pb = (C.c_void_p * n)(*[c.ptr.value for c in b_list])
        ms = C.c_float()
        _chk(lib().refx_time_hmult_set(self.ptr, pa, pb, n, int(rescale), warmup, iters, C.byref(ms)),
             "time HMult set")
        return ms.value

    def time_hrot(self, a, rot, iters, warmup=3):
        ms = C.c_float()
        _chk(lib().refx_time_hrot(self.ptr, a.ptr, rot, warmup, iters, C.byref(ms)), "time HRot")
        return ms.value

    def time_ntt_roundtrip(self, num_main, npoly, iters, warmup=3):
        ms = C.c_float()
        _chk(lib().refx_time_ntt_roundtrip(self.ptr, num_main, npoly, warmup, iters, C.byref(ms)), "time NTT")
        return ms.value

    def time_boot(self, c, iters, warmup=2, min_ks=False):
        ms = C.c_float()
        _chk(lib().refx_time_boot(self.ptr, c.ptr, int(min_ks), warmup, iters, C.byref(ms)), "time Boot")
        return ms.value


class RefCiphertext:
    def __init__(self, ctx):
        self.ctx = ctx
        self.ptr = C.c_void_p(lib().refx_ct_new())

    def free(self):
        if self.ptr is not None and self.ptr.value:
            lib().refx_ct_free(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def info(self):
        m, t, a, rx, ns = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        sc = C.c_double()
        lib().refx_ct_info(self.ptr, C.byref(m), C.byref(t), C.byref(a), C.byref(rx), C.byref(sc), C.byref(ns))
        return dict(num_main=m.value, num_ter=t.value, num_aux=a.value, has_rx=bool(rx.value), scale=sc.value,
                    num_slots=ns.value)

    def numpy(self):
        inf = self.info()
        rows = inf["num_main"] + inf["num_ter"] + inf["num_aux"]
        parts = [np.zeros((rows, self.ctx.n), dtype=np.uint32) for _ in range(3 if inf["has_rx"] else 2)]
        _chk(lib().refx_ct_export(self.ctx.ptr, self.ptr, parts[0].ctypes.data, parts[1].ctypes.data,
                                  parts[2].ctypes.data if len(parts) > 2 else None), "ct export")
        return parts


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


class RefContext64:
    """The reference's Context<uint64_t> (the 64-bit word path) on a
    parameter set with primes up to 2^62; keys and ciphertexts are imported
    ([np][N] uint64 host arrays)."""

    def __init__(self, params):
        p = json.loads(params) if isinstance(params, str) else params
        self.params = p
        lv = np.array([x for pair in p["level_config"] for x in pair], dtype=np.int32)
        main, aux = _u64(p["main_primes"]), _u64(p["auxiliary_primes"])
        ter = _u64(p.get("terminal_primes", []) or [0])
        n_ter = len(p.get("terminal_primes", []))
        add = p.get("additional_base", [0, 0])
        self._keep = (lv, main, aux, ter)
        self.ptr = C.c_void_p()
        _chk(lib().refx64_create(p["log_degree"], p["log_default_scale"], p["default_encryption_level"],
                                 len(p["level_config"]), lv.ctypes.data, main.ctypes.data, len(main),
                                 aux.ctypes.data, len(aux), ter.ctypes.data, n_ter, add[0], add[1],
                                 C.byref(self.ptr)), "create64")
        self.n = 1 << p["log_degree"]

    def close(self):
        if getattr(self, "ptr", None) is not None and self.ptr.value:
            lib().refx64_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def ntt(self, np_, data, inverse=False, mont=False):
        """NTT / INTT of polynomials [count][rows][N] over NPInfo np_ = (main, ter, aux)."""
        d = _u64(data).copy()
        count = d.shape[0] if d.ndim == 3 else 1
        _chk(lib().refx64_ntt(self.ptr, np_[0], np_[1], np_[2], d.ctypes.data, count, int(inverse), int(mont)),
             "ntt64")
        return d

    def modup(self, level, src, beta, rows_out):
        s = _u64(src)
        out = np.zeros((beta, rows_out, self.n), dtype=np.uint64)
        _chk(lib().refx64_modup(self.ptr, level, s.ctypes.data, out.ctypes.data), "modup64")
        return out

    def moddown(self, level, kind, src, rows_out):
        s = _u64(src)
        out = np.zeros((rows_out, self.n), dtype=np.uint64)
        _chk(lib().refx64_moddown(self.ptr, level, kind, s.ctypes.data, out.ctypes.data), "moddown64")
        return out

    def hmult(self, level, a, b, key, rescale, rows_out):
        a0, a1, b0, b1 = (_u64(x) for x in (a[0], a[1], b[0], b[1]))
        kb, ka = _u64(key[0]), _u64(key[1])
        ob = np.zeros((rows_out, self.n), dtype=np.uint64)
        oa = np.zeros_like(ob)
        _chk(lib().refx64_hmult(self.ptr, level, a0.ctypes.data, a1.ctypes.data, b0.ctypes.data, b1.ctypes.data,
                                kb.shape[0], kb.ctypes.data, ka.ctypes.data, int(rescale), ob.ctypes.data,
                                oa.ctypes.data), "hmult64")
        return ob, oa

    def hrot(self, level, a, key, rot, rows_out):
        a0, a1 = _u64(a[0]), _u64(a[1])
        kb, ka = _u64(key[0]), _u64(key[1])
        ob = np.zeros((rows_out, self.n), dtype=np.uint64)
        oa = np.zeros_like(ob)
        _chk(lib().refx64_hrot(self.ptr, level, a0.ctypes.data, a1.ctypes.data, kb.shape[0], kb.ctypes.data,
                               ka.ctypes.data, rot, ob.ctypes.data, oa.ctypes.data), "hrot64")
        return ob, oa

    def hconj(self, level, a, key, rows_out):
        a0, a1 = _u64(a[0]), _u64(a[1])
        kb, ka = _u64(key[0]), _u64(key[1])
        ob = np.zeros((rows_out, self.n), dtype=np.uint64)
        oa = np.zeros_like(ob)
        _chk(lib().refx64_hconj(self.ptr, level, a0.ctypes.data, a1.ctypes.data, kb.shape[0], kb.ctypes.data,
                                ka.ctypes.data, ob.ctypes.data, oa.ctypes.data), "hconj64")
        return ob, oa

    def op(self, name, level, a, b=None, key=None, arg=0, scale=0.0, value=0.0):
        """Context<uint64_t>::<name> on imported ciphertexts a (and b), each
        (bx, ax) or (bx, ax, rx) at `level`, and an imported key (kb, ka);
        returns the result's parts, rx included when it has one."""
        a = [_u64(x) for x in a]
        b = [_u64(x) for x in b] if b is not None else None
        ptr = lambda parts, i: parts[i].ctypes.data if parts is not None and len(parts) > i else None  # noqa: E731
        kb, ka = (_u64(key[0]), _u64(key[1])) if key is not None else (None, None)
        rows = a[0].shape[0]
        ob = np.zeros((rows, self.n), dtype=np.uint64)
        oa, orx = np.zeros_like(ob), np.zeros_like(ob)
        info = np.zeros(3, dtype=np.int32)
        _chk(lib().refx64_op(self.ptr, name.encode(), level, ptr(a, 0), ptr(a, 1), ptr(a, 2), ptr(b, 0), ptr(b, 1),
                             ptr(b, 2), kb.shape[0] if kb is not None else 0,
                             kb.ctypes.data if kb is not None else None, ka.ctypes.data if ka is not None else None,
                             int(arg), float(scale), float(value), ob.ctypes.data, oa.ctypes.data, orx.ctypes.data,
                             info.ctypes.data), "op64 " + name)
        r = int(info[0] + info[1])
        return (ob[:r], oa[:r], orx[:r]) if info[2] else (ob[:r], oa[:r])

    def time_hmult(self, level, a, b, key, rescale=True, warmup=3, iters=20):
        """Device milliseconds per HMult of the reference's 64-bit build."""
        a0, a1, b0, b1 = (_u64(x) for x in (a[0], a[1], b[0], b[1]))
        kb, ka = _u64(key[0]), _u64(key[1])
        ms = C.c_float()
        _chk(lib().refx64_time_hmult(self.ptr, level, a0.ctypes.data, a1.ctypes.data, b0.ctypes.data,
                                     b1.ctypes.data, kb.shape[0], kb.ctypes.data, ka.ctypes.data, int(rescale),
                                     warmup, iters, C.byref(ms)), "time_hmult64")
        return ms.value
