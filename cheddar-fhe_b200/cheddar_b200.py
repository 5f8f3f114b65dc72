"""Python binding of the B200 CKKS evaluation core (libcheddar_b200.so).

Mirrors the reference's server-side C++ API (scale-snu/cheddar-fhe,
include/core/Context.h, include/core/Container.h): a Context created from
the parameter JSON, device Ciphertexts, EvaluationKeys, and the evaluator
calls HMult / HRot / HConj / Relinearize / Rescale / ... with the same
argument meaning.  Everything runs in the CUDA library; this module only
marshals arguments.  It raises if the library is missing — there is no CPU
fallback.
"""
import ctypes as C
import json
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcheddar_b200.so")
PARAM_DIR = os.path.join(_HERE, "params")

CHD_MODDOWN, CHD_RESCALE, CHD_MODDOWN_RESCALE = 0, 1, 2
BCONV_CUDA_CORE, BCONV_TENSOR_CORE = 0, 1   # chd_bconv_batch engines
BCONV_AUTO = 2                                # Context.ks_engine only: autotuned per launch shape
BCONV_TENSOR_CORE_WIDE = 3                    # Context.ks_engine only: tensor cores, 256-thread tiles (K <= 12)

# stages of the fused N = 2^16 key switch (chd_stage_times), in launch order
KS_STAGE_NAMES = ("modup_inv_rows", "modup_cols", "ks_rows", "moddown_cols", "fwd_rows_epilogue")
KS_STAGES = len(KS_STAGE_NAMES)

_lib = None


class CheddarError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cheddar error {code}: {msg}")
        self.code = code


def build():
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE, "-j8"], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}`")
    L = C.CDLL(LIB_PATH)
    vp, i, d, u32p, i32p = C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p
    pp = C.POINTER(C.c_void_p)
    sig = {
        "chd_last_error": (C.c_char_p, []),
        "chd_context_create_json": (i, [C.c_char_p, i, pp]),
        "chd_context_create": (i, [i, d, i, i32p, i, u32p, i, u32p, i, u32p, i, i, i, i, pp]),
        "chd_context_destroy": (None, [vp]),
        "chd_context_set_stream": (i, [vp, vp]),
        "chd_context_synchronize": (i, [vp]),
        "chd_stage_timing": (i, [vp, i]),
        "chd_set_ks_engine": (i, [vp, i]),
        "chd_copy": (i, [vp, vp, vp]),
        "chd_mult_unsafe": (i, [vp, vp, vp, vp, i]),
        "chd_mult_unsafe_const": (i, [vp, vp, vp, vp, i, d, i]),
        "chd_mad_unsafe": (i, [vp, vp, vp, vp, i, d]),
        "chd_permute": (i, [vp, vp, vp, i]),
        "chd_permute_conjugate": (i, [vp, vp, vp]),
        "chd_hconj_add": (i, [vp, vp, vp, vp, vp]),
        "chd_level_down": (i, [vp, vp, vp, i]),
        "chd_mult_key_no_moddown": (i, [vp, vp, vp, vp]),
        "chd_mult_unsafe_compatible": (i, [vp, i, i]),
        "chd_add_plain": (i, [vp, vp, vp, vp, d]),
        "chd_sub_plain": (i, [vp, vp, vp, vp, d]),
        "chd_sub_const": (i, [vp, vp, vp, u32p]),
        "chd_sub_plain_ct": (i, [vp, vp, vp, d, vp]),
        "chd_sub_const_ct": (i, [vp, vp, u32p, d, vp]),
        "chd_mult_unsafe_plain": (i, [vp, vp, vp, vp, i, i, d, i]),
        "chd_get_ks_engine": (i, [vp]),
        "chd_set_stream_split": (i, [vp, i]),
        "chd_get_stream_split": (i, [vp]),
        "chd_stage_times": (i, [vp, vp, vp]),
        "chd_level_np": (i, [vp, i, C.POINTER(i), C.POINTER(i)]),
        "chd_max_level": (i, [vp]),
        "chd_degree": (i, [vp]),
        "chd_alpha": (i, [vp]),
        "chd_num_q_primes": (i, [vp]),
        "chd_scale": (d, [vp, i]),
        "chd_rescale_prime_prod": (d, [vp, i]),
        "chd_prime_gidx": (i, [vp, i, i, i, i32p]),
        "chd_ct_create": (i, [vp, pp]),
        "chd_ct_destroy": (None, [vp]),
        "chd_ct_wrap": (i, [vp, i, i, i, i, d, i, vp, vp, vp, C.c_size_t, pp]),
        "chd_ct_import": (i, [vp, vp, i, i, i, i, d, i, vp, vp, vp, i]),
        "chd_ct_export": (i, [vp, vp, vp, vp, vp, i]),
        "chd_ct_info": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i),
                            C.POINTER(d), C.POINTER(i)]),
        "chd_ct_device_ptrs": (i, [vp, pp, pp, pp]),
        "chd_evk_create": (i, [vp, i, vp, vp, i, pp]),
        "chd_evk_destroy": (None, [vp]),
        "chd_add": (i, [vp, vp, vp, vp]),
        "chd_sub": (i, [vp, vp, vp, vp]),
        "chd_neg": (i, [vp, vp, vp]),
        "chd_mult": (i, [vp, vp, vp, vp]),
        "chd_mult_const": (i, [vp, vp, vp, u32p, d]),
        "chd_add_const": (i, [vp, vp, vp, u32p]),
        "chd_mult_plain": (i, [vp, vp, vp, vp, d]),
        "chd_mult_imaginary_unit": (i, [vp, vp, vp]),
        "chd_rescale": (i, [vp, vp, vp]),
        "chd_relinearize": (i, [vp, vp, vp, vp]),
        "chd_relinearize_rescale": (i, [vp, vp, vp, vp]),
        "chd_mult_key": (i, [vp, vp, vp, vp]),
        "chd_hmult": (i, [vp, vp, vp, vp, vp, i]),
        "chd_hmult_batch": (i, [vp, i, pp, pp, pp, vp, i]),
        "chd_hrot": (i, [vp, vp, vp, vp, i]),
        "chd_hconj": (i, [vp, vp, vp, vp]),
        "chd_hrot_add": (i, [vp, vp, vp, vp, vp, i]),
        "chd_hoisted_rotate": (i, [vp, vp, i, i32p, pp, pp]),
        "chd_moddown": (i, [vp, vp, vp]),
        "chd_ntt": (i, [vp, i, i, i, vp, i, i]),
        "chd_intt": (i, [vp, i, i, i, vp, i, i]),
        "chd_modup_raw": (i, [vp, i, vp, vp]),
        "chd_moddown_raw": (i, [vp, i, i, vp, vp, i]),
        "chd_bconv_raw": (i, [vp, vp, i32p, i, i32p, i, vp]),
        "chd_bconv_batch": (i, [vp, i, i, vp, i32p, i, i32p, i, vp]),
        "chd_debug_stall_tensor_waits": (i, [vp, i]),
        "chd_decode": (i, [vp, i, C.c_double, vp, i, vp, vp]),
        "chd_evk_info": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)]),
        "chd_ks_tuned_shapes": (i, [vp, i]),
        "chd_ks_rows_tuned_shapes": (i, [vp, i]),
        "chd_moddown_batch": (i, [vp, i, vp, vp]),
        "chd_ct_serialize": (i, [vp, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)]),
        "chd_ct_deserialize": (i, [vp, vp, vp, C.c_size_t]),
        "chd_evk_serialize": (i, [vp, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)]),
        "chd_evk_deserialize": (i, [vp, vp, C.c_size_t, pp]),
        "chd_evk_export": (i, [vp, vp, vp, vp, i]),
        "chd_client_create": (i, [vp, C.c_uint64, pp]),
        "chd_client_destroy": (None, [vp]),
        "chd_client_secret": (i, [vp, vp, i, vp]),
        "chd_client_mult_key": (i, [vp, vp, pp]),
        "chd_client_rotation_key": (i, [vp, vp, i, pp]),
        "chd_client_conjugation_key": (i, [vp, vp, pp]),
        "chd_client_sse_keys": (i, [vp, vp, pp, pp]),
        "chd_client_encrypt": (i, [vp, vp, C.c_uint64, i, C.c_double, i, vp, vp]),
        "chd_client_decrypt": (i, [vp, vp, vp, vp]),
        "chd_encode": (i, [vp, i, d, vp, vp, i, i, vp, C.POINTER(i)]),
        "chd_encode_const": (i, [vp, i, d, d, i, vp]),
        "chd_modup_to_max": (i, [vp, vp, vp, vp]),
        "chd_evk_map_create": (i, [vp, pp]),
        "chd_evk_map_destroy": (None, [vp]),
        "chd_evk_map_set_rotation": (i, [vp, i, vp]),
        "chd_evk_map_set_conjugation": (i, [vp, vp]),
        "chd_evk_map_set_mult": (i, [vp, vp]),
        "chd_evk_map_set_dense_to_sparse": (i, [vp, vp]),
        "chd_evk_map_set_sparse_to_dense": (i, [vp, vp]),
        "chd_evk_create_np": (i, [vp, i, i, i, i, vp, vp, i, pp]),
        "chd_lintrans_create": (i, [vp, i, i, vp, vp, vp, i, d, i, i, i, i, pp]),
        "chd_lintrans_destroy": (None, [vp]),
        "chd_lintrans_rotations": (i, [vp, i, vp, i, C.POINTER(i)]),
        "chd_lintrans_num_pts": (i, [vp, C.POINTER(i)]),
        "chd_lintrans_pt": (i, [vp, i, C.POINTER(i), C.POINTER(i), vp, vp]),
        "chd_lintrans_evaluate": (i, [vp, vp, vp, vp, vp, i]),
        "chd_poly_create": (i, [vp, vp, i, i, d, d, i, pp]),
        "chd_evalmod_create": (i, [vp, i, vp, i, i, i, pp, C.POINTER(d), C.POINTER(d)]),
        "chd_program_destroy": (None, [vp]),
        "chd_program_json": (i, [vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "chd_program_run": (i, [vp, vp, vp, vp, vp]),
        "chd_boot_mod_coefficients": (i, [vp, i]),
        "chd_boot_create": (i, [vp, i, i, i, i, pp]),
        "chd_boot_create_variant": (i, [vp, i, i, i, i, i, pp]),
        "chd_boot_run_batch": (i, [vp, vp, i, pp, pp, vp, i]),
        "chd_boot_destroy": (None, [vp]),
        "chd_boot_rotations": (i, [vp, i, vp, i, C.POINTER(i)]),
        "chd_boot_levels": (i, [vp, vp, vp]),
        "chd_boot_json": (i, [vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "chd_boot_lt_info": (i, [vp, i, C.POINTER(i), C.POINTER(d), C.POINTER(i), C.POINTER(i)]),
        "chd_boot_lt_pt": (i, [vp, i, i, C.POINTER(i), C.POINTER(i), vp, vp]),
        "chd_boot_run": (i, [vp, vp, vp, vp, vp, i]),
        "chd_graph_begin": (i, [vp]),
        "chd_graph_end": (i, [vp, pp]),
        "chd_graph_launch": (i, [vp, vp]),
        "chd_graph_destroy": (None, [vp]),
        "chd64_context_create_json": (i, [C.c_char_p, i, pp]),
        "chd64_context_destroy": (None, [vp]),
        "chd64_context_synchronize": (i, [vp]),
        "chd64_context_set_stream": (i, [vp, vp]),
        "chd64_max_level": (i, [vp]),
        "chd64_alpha": (i, [vp]),
        "chd64_level_np": (i, [vp, i, C.POINTER(i), C.POINTER(i)]),
        "chd64_primes": (i, [vp, vp, i]),
        "chd64_ntt": (i, [vp, i, i, i, vp, i, i, i]),
        "chd64_modup_raw": (i, [vp, i, vp, vp]),
        "chd64_moddown_raw": (i, [vp, i, i, vp, vp, i]),
        "chd64_ct_create": (i, [vp, pp]),
        "chd64_ct_destroy": (None, [vp]),
        "chd64_ct_import": (i, [vp, vp, i, d, i, vp, vp, i]),
        "chd64_ct_export": (i, [vp, vp, vp, vp]),
        "chd64_ct_info": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(d), C.POINTER(i)]),
        "chd64_evk_create": (i, [vp, i, vp, vp, i, pp]),
        "chd64_evk_destroy": (None, [vp]),
        "chd64_hmult": (i, [vp, vp, vp, vp, vp, i]),
        "chd64_hrot": (i, [vp, vp, vp, vp, i]),
        "chd64_rescale": (i, [vp, vp, vp]),
        "chd64_hconj": (i, [vp, vp, vp, vp]),
        "chd64_ct_set_rx": (i, [vp, vp, vp, i]),
        "chd64_ct_export_rx": (i, [vp, vp, vp]),
        "chd64_ct_has_rx": (i, [vp]),
        "chd64_scale": (C.c_double, [vp, i]),
        "chd64_encode_const": (i, [vp, i, C.c_double, C.c_double, i, vp]),
        "chd64_copy": (i, [vp, vp, vp]),
        "chd64_neg": (i, [vp, vp, vp]),
        "chd64_mult_imaginary_unit": (i, [vp, vp, vp]),
        "chd64_add": (i, [vp, vp, vp, vp]),
        "chd64_sub": (i, [vp, vp, vp, vp]),
        "chd64_mult": (i, [vp, vp, vp, vp]),
        "chd64_relinearize": (i, [vp, vp, vp, vp, i]),
        "chd64_mult_key": (i, [vp, vp, vp, vp]),
        "chd64_permute": (i, [vp, vp, vp, i, i]),
        "chd64_hrot_add": (i, [vp, vp, vp, vp, vp, i]),
        "chd64_hconj_add": (i, [vp, vp, vp, vp, vp]),
        "chd64_mult_const": (i, [vp, vp, vp, vp, C.c_double]),
        "chd64_add_const": (i, [vp, vp, vp, vp]),
        "chd64_level_down": (i, [vp, vp, vp, i]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise CheddarError(rc, lib().chd_last_error().decode())


def _ptr(a):
    """Device or host pointer of a numpy array or torch tensor."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def ks_tuned_shapes():
    """The column-pass autotuner's choices in this process: one dict per
    launch shape (largest source count K, jobs, largest target count M) with
    the engine (0 CUDA cores, 1 tensor cores) and the target split."""
    n = lib().chd_ks_tuned_shapes(None, 0)
    out = (C.c_int * (6 * max(1, n)))()
    n = lib().chd_ks_tuned_shapes(out, n)
    return [dict(device=out[6 * i], K=out[6 * i + 1], jobs=out[6 * i + 2], M=out[6 * i + 3],
                 engine=out[6 * i + 4], split=out[6 * i + 5]) for i in range(n)]


def ks_rows_tuned_shapes():
    """The key-switch row pass's autotuned choices in this process: one dict
    per launch shape with its `variant` (0 loads where used at 3 CTAs per
    SM, 1 loads ahead at 2, 2 loads where used at 4) and `prefetch` True for
    variant 1."""
    n = lib().chd_ks_rows_tuned_shapes(None, 0)
    out = (C.c_int * (5 * max(1, n)))()
    n = lib().chd_ks_rows_tuned_shapes(out, n)
    return [dict(device=out[5 * i], cts=out[5 * i + 1], rows=out[5 * i + 2], mode=out[5 * i + 3],
                 variant=out[5 * i + 4], prefetch=out[5 * i + 4] == 1) for i in range(n)]


def load_params(name_or_path):
    path = name_or_path
    if not os.path.exists(path):
        path = os.path.join(PARAM_DIR, name_or_path)
    with open(path) as f:
        return f.read()


class Context:
    """Context<uint32_t>::Create(Parameter) (include/core/Context.h:70)."""

    def __init__(self, json_text, device=0):
        self.ptr = C.c_void_p()
        _check(lib().chd_context_create_json(json_text.encode(), device, C.byref(self.ptr)))
        L = lib()
        self.max_level = L.chd_max_level(self.ptr)
        self.n = L.chd_degree(self.ptr)
        self.alpha = L.chd_alpha(self.ptr)
        self.L = L.chd_num_q_primes(self.ptr)

    @classmethod
    def from_params(cls, name_or_path, device=0):
        return cls(load_params(name_or_path), device)

    def close(self):
        if getattr(self, "ptr", None) and self.ptr.value:
            lib().chd_context_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        _check(lib().chd_context_set_stream(self.ptr, stream_handle))

    def synchronize(self):
        _check(lib().chd_context_synchronize(self.ptr))

    def graph_begin(self):
        """Start capturing the GPU work of the following calls (see Graph)."""
        _check(lib().chd_graph_begin(self.ptr))

    def graph_end(self):
        g = C.c_void_p()
        _check(lib().chd_graph_end(self.ptr, C.byref(g)))
        return Graph(self, g)

    @property
    def ks_engine(self):
        """Base-conversion engine of the key-switching and rescaling paths:
        BCONV_CUDA_CORE, BCONV_TENSOR_CORE or BCONV_AUTO (the faster of the
        two per launch shape, measured on first use); residues are
        bit-identical."""
        return lib().chd_get_ks_engine(self.ptr)

    @ks_engine.setter
    def ks_engine(self, engine):
        _check(lib().chd_set_ks_engine(self.ptr, int(engine)))

    @property
    def stream_split(self):
        """Whether a fused key switch of two or more ciphertexts runs its two
        halves on two streams of the context (on by default; identical
        residues either way)."""
        return bool(lib().chd_get_stream_split(self.ptr))

    @stream_split.setter
    def stream_split(self, on):
        _check(lib().chd_set_stream_split(self.ptr, 1 if on else 0))

    def stage_timing(self, enable):
        """Start (clearing earlier records) or stop device timing of the fused
        key-switch stages."""
        _check(lib().chd_stage_timing(self.ptr, 1 if enable else 0))

    def stage_times(self):
        """{stage: (device ms, launches)} summed since stage_timing(True)."""
        ms = (C.c_double * KS_STAGES)()
        nl = (C.c_int * KS_STAGES)()
        _check(lib().chd_stage_times(self.ptr, ms, nl))
        return {name: (ms[i], nl[i]) for i, name in enumerate(KS_STAGE_NAMES)}

    def level_np(self, level):
        m, t = C.c_int(), C.c_int()
        _check(lib().chd_level_np(self.ptr, level, C.byref(m), C.byref(t)))
        return m.value, t.value

    def num_q(self, level):
        m, t = self.level_np(level)
        return m + t

    def scale(self, level):
        return lib().chd_scale(self.ptr, level)

    def rescale_prime_prod(self, level):
        return lib().chd_rescale_prime_prod(self.ptr, level)

    def level_of(self, num_main, num_ter):
        """The level whose q primes are (num_main, num_ter)."""
        for lv in range(-1, self.max_level + 1):
            if self.level_np(lv) == (num_main, num_ter):
                return lv
        raise CheddarError(2, f"no level holds {num_main} main and {num_ter} terminal primes")

    def gidx(self, num_main, num_ter, num_aux):
        out = np.zeros(256, dtype=np.int32)
        k = lib().chd_prime_gidx(self.ptr, num_main, num_ter, num_aux, out.ctypes.data)
        return out[:k].copy()

    # ---- containers ----
    def ciphertext(self):
        return Ciphertext(self)

    def import_ct(self, level, parts, scale=1.0, num_slots=None, num_aux=0, on_device=False):
        ct = Ciphertext(self)
        ct.load(level, parts, scale, num_slots, num_aux, on_device)
        return ct

    def wrap_ct(self, level, parts, scale=1.0, num_slots=None, num_aux=0):
        """Ciphertext over caller-owned device buffers (torch tensors)."""
        m, t = self.level_np(level)
        rows = m + t + num_aux
        words = min(int(p.numel()) for p in parts)
        assert words >= rows * self.n
        ct = Ciphertext.__new__(Ciphertext)
        ct.ctx = self
        ct.ptr = C.c_void_p()
        ct._keep = parts
        rx = _ptr(parts[2]) if len(parts) > 2 else None
        _check(lib().chd_ct_wrap(self.ptr, m, t, num_aux, int(len(parts) > 2), scale,
                                 num_slots or self.n // 2, _ptr(parts[0]), _ptr(parts[1]), rx,
                                 words, C.byref(ct.ptr)))
        return ct

    def load_ct(self, data):
        """A ciphertext from bytes written by Ciphertext.serialize."""
        ct = Ciphertext(self)
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(lib().chd_ct_deserialize(self.ptr, ct.ptr, buf, len(data)))
        return ct

    def load_evk(self, data):
        """An evaluation key from bytes written by EvaluationKey.serialize."""
        k = EvaluationKey.__new__(EvaluationKey)
        k.ctx = self
        k.ptr = C.c_void_p()
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(lib().chd_evk_deserialize(self.ptr, buf, len(data), C.byref(k.ptr)))
        return k

    def evk(self, bx, ax, on_device=False):
        return EvaluationKey(self, bx, ax, on_device)

    # ---- evaluator (Context.cpp of the reference) ----
    def _new(self, res):
        return res if res is not None else Ciphertext(self)

    def Add(self, a, b, res=None):
        res = self._new(res)
        _check(lib().chd_add(self.ptr, res.ptr, a.ptr, b.ptr))
        return res

    def Sub(self, a, b, res=None):
        res = self._new(res)
        _check(lib().chd_sub(self.ptr, res.ptr, a.ptr, b.ptr))
        return res

    def Neg(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_neg(self.ptr, res.ptr, a.ptr))
        return res

    def Mult(self, a, b, res=None):
        res = self._new(res)
        _check(lib().chd_mult(self.ptr, res.ptr, a.ptr, b.ptr))
        return res

    def MultConst(self, a, cx, const_scale, res=None):
        res = self._new(res)
        cx = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_mult_const(self.ptr, res.ptr, a.ptr, cx.ctypes.data, const_scale))
        return res

    def AddConst(self, a, cx, res=None):
        res = self._new(res)
        cx = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_add_const(self.ptr, res.ptr, a.ptr, cx.ctypes.data))
        return res

    def SubConst(self, a, cx, res=None):
        """a - c (Context::Sub(Ct, Ct, Const))."""
        res = self._new(res)
        cx = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_sub_const(self.ptr, res.ptr, a.ptr, cx.ctypes.data))
        return res

    def SubConstCt(self, cx, const_scale, b, res=None):
        """c - b (Context::Sub(Ct, Const, Ct))."""
        res = self._new(res)
        cx = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_sub_const_ct(self.ptr, res.ptr, cx.ctypes.data, float(const_scale), b.ptr))
        return res

    def MultPlain(self, a, pt, pt_scale, res=None):
        """a (.) pt (Context::Mult(Ct, Ct, Pt)); pt: device residues over a's
        primes, as encode() gives them."""
        res = self._new(res)
        _check(lib().chd_mult_plain(self.ptr, res.ptr, a.ptr, _ptr(pt), float(pt_scale)))
        return res

    def AddPlain(self, a, pt, pt_scale, res=None):
        """a + pt (Context::Add(Ct, Ct, Pt)); the scales must match."""
        res = self._new(res)
        _check(lib().chd_add_plain(self.ptr, res.ptr, a.ptr, _ptr(pt), float(pt_scale)))
        return res

    def SubPlain(self, a, pt, pt_scale, res=None):
        """a - pt (Context::Sub(Ct, Ct, Pt))."""
        res = self._new(res)
        _check(lib().chd_sub_plain(self.ptr, res.ptr, a.ptr, _ptr(pt), float(pt_scale)))
        return res

    def SubPlainCt(self, pt, pt_scale, b, res=None):
        """pt - b (Context::Sub(Ct, Pt, Ct))."""
        res = self._new(res)
        _check(lib().chd_sub_plain_ct(self.ptr, res.ptr, _ptr(pt), float(pt_scale), b.ptr))
        return res

    def MultUnsafePlain(self, a, pt, pt_level, pt_scale, pt_num_aux=0, level=-1, res=None):
        """a (.) pt at `level` (-1: the lower level), reading both past their
        extra terminal primes (Context::MultUnsafe(Ct, Ct, Pt, level))."""
        res = self._new(res)
        _check(lib().chd_mult_unsafe_plain(self.ptr, res.ptr, a.ptr, _ptr(pt), pt_level, pt_num_aux,
                                           float(pt_scale), level))
        return res

    def MultImaginaryUnit(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_mult_imaginary_unit(self.ptr, res.ptr, a.ptr))
        return res

    def Rescale(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_rescale(self.ptr, res.ptr, a.ptr))
        return res

    def Relinearize(self, a, key, res=None):
        res = self._new(res)
        _check(lib().chd_relinearize(self.ptr, res.ptr, a.ptr, key.ptr))
        return res

    def RelinearizeRescale(self, a, key, res=None):
        res = self._new(res)
        _check(lib().chd_relinearize_rescale(self.ptr, res.ptr, a.ptr, key.ptr))
        return res

    def MultKey(self, a, key, res=None):
        res = self._new(res)
        _check(lib().chd_mult_key(self.ptr, res.ptr, a.ptr, key.ptr))
        return res

    def HMult(self, a, b, mult_key, rescale=True, res=None):
        res = self._new(res)
        _check(lib().chd_hmult(self.ptr, res.ptr, a.ptr, b.ptr, mult_key.ptr, int(rescale)))
        return res

    def HMultBatch(self, a_list, b_list, mult_key, rescale=True, res_list=None):
        n = len(a_list)
        res_list = res_list or [Ciphertext(self) for _ in range(n)]
        arr = lambda xs: (C.c_void_p * n)(*[x.ptr.value for x in xs])
        _check(lib().chd_hmult_batch(self.ptr, n, arr(res_list), arr(a_list), arr(b_list),
                                     mult_key.ptr, int(rescale)))
        return res_list

    def HRot(self, a, rot_key, rot_dist, res=None):
        res = self._new(res)
        _check(lib().chd_hrot(self.ptr, res.ptr, a.ptr, rot_key.ptr, rot_dist))
        return res

    def HConj(self, a, conj_key, res=None):
        res = self._new(res)
        _check(lib().chd_hconj(self.ptr, res.ptr, a.ptr, conj_key.ptr))
        return res

    def HRotAdd(self, a, b, rot_key, rot_dist, res=None):
        res = self._new(res)
        _check(lib().chd_hrot_add(self.ptr, res.ptr, a.ptr, b.ptr, rot_key.ptr, rot_dist))
        return res

    def Copy(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_copy(self.ptr, res.ptr, a.ptr))
        return res

    def MultUnsafe(self, a, b, level=-1, res=None):
        """Tensor product at `level` (-1: the lower input level)."""
        res = self._new(res)
        _check(lib().chd_mult_unsafe(self.ptr, res.ptr, a.ptr, b.ptr, level))
        return res

    def MultUnsafeConst(self, a, cx, const_level, const_scale, level=-1, res=None):
        """a times a constant (cx: Montgomery residues over const_level's q
        primes, as encode_const gives them) at `level`."""
        res = self._new(res)
        c = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_mult_unsafe_const(self.ptr, res.ptr, a.ptr, c.ctypes.data, const_level, float(const_scale),
                                           level))
        return res

    def MadUnsafe(self, res, a, cx, const_level, const_scale):
        """res += a times a constant."""
        c = np.ascontiguousarray(cx, dtype=np.uint32)
        _check(lib().chd_mad_unsafe(self.ptr, res.ptr, a.ptr, c.ctypes.data, const_level, float(const_scale)))
        return res

    def Permute(self, a, rot_dist, res=None):
        res = self._new(res)
        _check(lib().chd_permute(self.ptr, res.ptr, a.ptr, rot_dist))
        return res

    def PermuteConjugate(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_permute_conjugate(self.ptr, res.ptr, a.ptr))
        return res

    def HConjAdd(self, a, b, conj_key, res=None):
        res = self._new(res)
        _check(lib().chd_hconj_add(self.ptr, res.ptr, a.ptr, b.ptr, conj_key.ptr))
        return res

    def LevelDown(self, a, target_level, res=None):
        res = self._new(res)
        _check(lib().chd_level_down(self.ptr, res.ptr, a.ptr, target_level))
        return res

    def MultKeyNoModDown(self, a, key, res=None):
        """Key switch of a left in the extended basis (relinearisation when a
        carries rx, else the key switch of a rotation)."""
        res = self._new(res)
        _check(lib().chd_mult_key_no_moddown(self.ptr, res.ptr, a.ptr, key.ptr))
        return res

    def IsMultUnsafeCompatible(self, level1, level2):
        r = lib().chd_mult_unsafe_compatible(self.ptr, level1, level2)
        if r < 0:
            raise CheddarError(1, "IsMultUnsafeCompatible: invalid level")
        return bool(r)

    def HoistedRotate(self, a, rot_keys, rot_dists, outs=None):
        n = len(rot_dists)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        d = np.asarray(rot_dists, dtype=np.int32)
        keys = (C.c_void_p * n)(*[k.ptr.value for k in rot_keys])
        outp = (C.c_void_p * n)(*[o.ptr.value for o in outs])
        _check(lib().chd_hoisted_rotate(self.ptr, a.ptr, n, d.ctypes.data, keys, outp))
        return outs

    def ModDown(self, a, res=None):
        res = self._new(res)
        _check(lib().chd_moddown(self.ptr, res.ptr, a.ptr))
        return res

    def ModDownBatch(self, cts, res_list=None):
        """ModDown of every ciphertext of `cts` (one level, Q u P) in one
        pipeline; equals ModDown on each."""
        res_list = res_list if res_list is not None else [Ciphertext(self) for _ in cts]
        n = len(cts)
        ins = (C.c_void_p * n)(*[c.ptr.value for c in cts])
        outs = (C.c_void_p * n)(*[r.ptr.value for r in res_list])
        _check(lib().chd_moddown_batch(self.ptr, n, outs, ins))
        return res_list

    # ---- raw device-buffer kernels (parity entry points) ----
    def ntt_raw(self, num_main, num_ter, num_aux, dev_ptr, mont=False, count=1):
        _check(lib().chd_ntt(self.ptr, num_main, num_ter, num_aux, _ptr(dev_ptr), int(mont), count))

    def intt_raw(self, num_main, num_ter, num_aux, dev_ptr, mont=True, count=1):
        _check(lib().chd_intt(self.ptr, num_main, num_ter, num_aux, _ptr(dev_ptr), int(mont), count))

    def modup_raw(self, level, src, dst):
        _check(lib().chd_modup_raw(self.ptr, level, _ptr(src), _ptr(dst)))

    def moddown_raw(self, level, kind, src, dst, npoly=1):
        _check(lib().chd_moddown_raw(self.ptr, level, kind, _ptr(src), _ptr(dst), npoly))

    def bconv_raw(self, xt, src_gidx, dst_gidx, out):
        s = np.ascontiguousarray(src_gidx, dtype=np.int32)
        d = np.ascontiguousarray(dst_gidx, dtype=np.int32)
        _check(lib().chd_bconv_raw(self.ptr, _ptr(xt), s.ctypes.data, len(s), d.ctypes.data, len(d),
                                   _ptr(out)))

    def encode(self, level, scale, msg, num_aux=0, out=None):
        """Encoder::Encode: complex slots -> device plaintext (torch int32
        [num_q(level) + num_aux][N], evaluation domain, Montgomery form)."""
        import torch
        msg = np.asarray(msg, dtype=np.complex128)
        re = np.ascontiguousarray(msg.real)
        im = np.ascontiguousarray(msg.imag)
        if out is None:
            out = torch.empty((self.num_q(level) + num_aux, self.n), dtype=torch.int32, device="cuda")
        ns = C.c_int()
        _check(lib().chd_encode(self.ptr, level, scale, re.ctypes.data, im.ctypes.data, len(msg), num_aux,
                                _ptr(out), C.byref(ns)))
        return out

    def decode(self, level, scale, pt, num_slots=None):
        """Encoder::Decode: device plaintext (torch int32 [num_q(level)][N],
        evaluation domain, Montgomery form) -> num_slots complex slots."""
        ns = num_slots or self.n // 2
        re = np.zeros(ns)
        im = np.zeros(ns)
        _check(lib().chd_decode(self.ptr, level, scale, _ptr(pt), ns, re.ctypes.data, im.ctypes.data))
        return re + 1j * im

    def encode_const(self, level, scale, value, num_aux=0):
        """Encoder::EncodeConstant: Montgomery residues per prime (host)."""
        out = np.zeros(self.num_q(level) + num_aux, dtype=np.uint32)
        _check(lib().chd_encode_const(self.ptr, level, scale, value, num_aux, out.ctypes.data))
        return out

    def ModUpToMax(self, a, res=None, keys=None):
        """BootContext::ModUpToMax; keys (EvkMap) with the dense-to-sparse and
        sparse-to-dense keys under sparse-secret encapsulation."""
        res = res if res is not None else Ciphertext(self)
        _check(lib().chd_modup_to_max(self.ptr, res.ptr, a.ptr, keys.ptr if keys is not None else None))
        return res

    def bconv_batch(self, xt, src_gidx, dst_gidx, out, engine=BCONV_CUDA_CORE, npoly=1):
        """Batched BConv of npoly polynomials ([npoly][K][N] int32 centred ->
        [npoly][M][N]); engine BCONV_CUDA_CORE or BCONV_TENSOR_CORE (tcgen05
        INT8 limb split), identical results.  Asynchronous on the context
        stream."""
        s = np.ascontiguousarray(src_gidx, dtype=np.int32)
        d = np.ascontiguousarray(dst_gidx, dtype=np.int32)
        _check(lib().chd_bconv_batch(self.ptr, engine, npoly, _ptr(xt), s.ctypes.data, len(s), d.ctypes.data,
                                     len(d), _ptr(out)))


class Graph:
    """A captured CUDA graph of library calls; launch() replays it on the
    context stream over the same buffers."""

    def __init__(self, ctx, ptr):
        self.ctx = ctx
        self.ptr = ptr

    def launch(self):
        _check(lib().chd_graph_launch(self.ctx.ptr, self.ptr))

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_graph_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass


class EvkMap:
    """EvkMap (include/core/EvkMap.h): keys by rotation index plus the
    conjugation and multiplication keys; holds references to the keys."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        self._keep = []
        _check(lib().chd_evk_map_create(ctx.ptr, C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_evk_map_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def set_rotation(self, r, key):
        self._keep.append(key)
        _check(lib().chd_evk_map_set_rotation(self.ptr, r, key.ptr))

    def set_conjugation(self, key):
        self._keep.append(key)
        _check(lib().chd_evk_map_set_conjugation(self.ptr, key.ptr))

    def set_mult(self, key):
        self._keep.append(key)
        _check(lib().chd_evk_map_set_mult(self.ptr, key.ptr))

    def set_dense_to_sparse(self, key):
        self._keep.append(key)
        _check(lib().chd_evk_map_set_dense_to_sparse(self.ptr, key.ptr))

    def set_sparse_to_dense(self, key):
        self._keep.append(key)
        _check(lib().chd_evk_map_set_sparse_to_dense(self.ptr, key.ptr))


class LinearTransform:
    """LinearTransform + HoistHandler (src/extension/LinearTransform.cpp,
    Hoist.cu): diagonals {index: complex[width]} encoded at pt_level."""

    def __init__(self, ctx, diags, pt_level, pt_scale, bs, gs=1, pre_rotation=0, additional_pt_rot=0):
        self.ctx = ctx
        idx = sorted(diags)
        width = len(diags[idx[0]])
        vals = np.stack([np.asarray(diags[i], dtype=np.complex128) for i in idx])
        re = np.ascontiguousarray(vals.real)
        im = np.ascontiguousarray(vals.imag)
        ia = np.ascontiguousarray(idx, dtype=np.int32)
        self.width = width
        self.ptr = C.c_void_p()
        _check(lib().chd_lintrans_create(ctx.ptr, width, len(idx), ia.ctypes.data, re.ctypes.data, im.ctypes.data,
                                         pt_level, pt_scale, bs, gs, pre_rotation, additional_pt_rot,
                                         C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_lintrans_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def rotations(self, min_ks=False):
        cnt = C.c_int()
        _check(lib().chd_lintrans_rotations(self.ptr, int(min_ks), None, 0, C.byref(cnt)))
        out = (C.c_int * max(1, cnt.value))()
        _check(lib().chd_lintrans_rotations(self.ptr, int(min_ks), out, cnt.value, C.byref(cnt)))
        return [out[i] for i in range(cnt.value)]

    def plaintexts(self):
        """[(giant step, baby step, message)] as compiled (after the swap)."""
        cnt = C.c_int()
        _check(lib().chd_lintrans_num_pts(self.ptr, C.byref(cnt)))
        res = []
        for i in range(cnt.value):
            g, b = C.c_int(), C.c_int()
            re = np.zeros(self.width)
            im = np.zeros(self.width)
            _check(lib().chd_lintrans_pt(self.ptr, i, C.byref(g), C.byref(b), re.ctypes.data, im.ctypes.data))
            res.append((g.value, b.value, re + 1j * im))
        return res

    def evaluate(self, ct, keys, res=None, min_ks=False):
        res = res if res is not None else Ciphertext(self.ctx)
        _check(lib().chd_lintrans_evaluate(self.ctx.ptr, self.ptr, res.ptr, ct.ptr, keys.ptr, int(min_ks)))
        return res


def boot_mod_coefficients():
    """BootParameter's EvalMod Chebyshev coefficients."""
    n = lib().chd_boot_mod_coefficients(None, 0)
    out = np.zeros(n)
    lib().chd_boot_mod_coefficients(out.ctypes.data, n)
    return out


class Program:
    """A compiled ciphertext program (EvalPoly / EvalMod)."""

    def __init__(self, ctx, ptr, start_scale=None, end_scale=None):
        self.ctx = ctx
        self.ptr = ptr
        self.start_scale = start_scale
        self.end_scale = end_scale

    @classmethod
    def poly(cls, ctx, coeffs, input_level, input_scale, target_scale, chebyshev=True):
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        p = C.c_void_p()
        _check(lib().chd_poly_create(ctx.ptr, c.ctypes.data, len(c), input_level, input_scale, target_scale,
                                     int(chebyshev), C.byref(p)))
        return cls(ctx, p, input_scale, target_scale)

    @classmethod
    def evalmod(cls, ctx, start_level, coeffs, num_double_angle=3, initial_K=2):
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        p = C.c_void_p()
        s0, s1 = C.c_double(), C.c_double()
        _check(lib().chd_evalmod_create(ctx.ptr, start_level, c.ctypes.data, len(c), num_double_angle, initial_K,
                                        C.byref(p), C.byref(s0), C.byref(s1)))
        return cls(ctx, p, s0.value, s1.value)

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_program_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def json(self):
        import json
        n = C.c_size_t()
        _check(lib().chd_program_json(self.ptr, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().chd_program_json(self.ptr, buf, n.value, C.byref(n)))
        return json.loads(buf.value.decode())

    def run(self, ct, keys, res=None):
        res = res if res is not None else Ciphertext(self.ctx)
        _check(lib().chd_program_run(self.ctx.ptr, self.ptr, res.ptr, ct.ptr, keys.ptr))
        return res


BOOT_NORMAL, BOOT_IMAGINARY_REMOVING, BOOT_MERGE_TWO_REAL = 0, 1, 2   # BootVariant


class BootContext:
    """BootContext prepared for `num_slots` (a power of two from 256 to N/2)
    and a BootVariant: CoeffToSlot, EvalMod, SlotToCoeff
    (src/extension/BootContext.cpp)."""

    def __init__(self, ctx, num_slots=None, num_cts_levels=4, num_stc_levels=3, log_message_ratio=5,
                 variant=BOOT_NORMAL):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        ns = num_slots if num_slots is not None else ctx.n // 2
        self.num_slots, self.variant = ns, variant
        _check(lib().chd_boot_create_variant(ctx.ptr, ns, variant, num_cts_levels, num_stc_levels,
                                             log_message_ratio, C.byref(self.ptr)))
        lv = (C.c_int * 5)()
        sc = (C.c_double * 5)()
        _check(lib().chd_boot_levels(self.ptr, lv, sc))
        self.cts_start, self.eval_mod_start, self.stc_start, self.end_level, self.log_scaleup = list(lv)
        self.cts_const, self.stc_const, self.eval_mod_start_scale, self.eval_mod_end_scale, self.final_scale = list(sc)

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_boot_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def rotations(self, min_ks=False):
        cnt = C.c_int()
        _check(lib().chd_boot_rotations(self.ptr, int(min_ks), None, 0, C.byref(cnt)))
        out = (C.c_int * max(1, cnt.value))()
        _check(lib().chd_boot_rotations(self.ptr, int(min_ks), out, cnt.value, C.byref(cnt)))
        return [out[i] for i in range(cnt.value)]

    def json(self):
        import json
        n = C.c_size_t()
        _check(lib().chd_boot_json(self.ptr, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().chd_boot_json(self.ptr, buf, n.value, C.byref(n)))
        return json.loads(buf.value.decode())

    def transforms(self):
        """[{level, scale, pts: [(gs, bs, message)]}] for CtS then StC."""
        res = []
        i = 0
        while True:
            lvl, sc, npts, w = C.c_int(), C.c_double(), C.c_int(), C.c_int()
            if lib().chd_boot_lt_info(self.ptr, i, C.byref(lvl), C.byref(sc), C.byref(npts), C.byref(w)) != 0:
                break
            pts = []
            for j in range(npts.value):
                g, b = C.c_int(), C.c_int()
                re = np.zeros(w.value)
                im = np.zeros(w.value)
                _check(lib().chd_boot_lt_pt(self.ptr, i, j, C.byref(g), C.byref(b), re.ctypes.data, im.ctypes.data))
                pts.append((g.value, b.value, re + 1j * im))
            res.append({"level": lvl.value, "scale": sc.value, "pts": pts})
            i += 1
        return res

    def Boot(self, ct, keys, res=None, min_ks=False):
        res = res if res is not None else Ciphertext(self.ctx)
        _check(lib().chd_boot_run(self.ctx.ptr, self.ptr, res.ptr, ct.ptr, keys.ptr, int(min_ks)))
        return res

    def BootBatch(self, cts, keys, res_list=None, min_ks=False):
        """Boot of every ciphertext in `cts` in one call, key switches and
        linear transforms batched across them; equals Boot on each."""
        res_list = res_list if res_list is not None else [Ciphertext(self.ctx) for _ in cts]
        n = len(cts)
        ins = (C.c_void_p * n)(*[c.ptr.value for c in cts])
        outs = (C.c_void_p * n)(*[r.ptr.value for r in res_list])
        _check(lib().chd_boot_run_batch(self.ctx.ptr, self.ptr, n, C.cast(outs, C.POINTER(C.c_void_p)),
                                        C.cast(ins, C.POINTER(C.c_void_p)), keys.ptr, int(min_ks)))
        return res_list


class Ciphertext:
    """Ciphertext<uint32_t> on the device (include/core/Container.h:131-175)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        _check(lib().chd_ct_create(ctx.ptr, C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_ct_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def load(self, level, parts, scale=1.0, num_slots=None, num_aux=0, on_device=False):
        m, t = self.ctx.level_np(level)
        num_slots = num_slots or self.ctx.n // 2
        if on_device:
            ps = [_ptr(p) for p in parts]
        else:
            self._host = [np.ascontiguousarray(p, dtype=np.uint32) for p in parts]
            ps = [p.ctypes.data for p in self._host]
        rx = ps[2] if len(ps) > 2 else None
        _check(lib().chd_ct_import(self.ctx.ptr, self.ptr, m, t, num_aux, int(len(ps) > 2), scale,
                                   num_slots, ps[0], ps[1], rx, int(on_device)))
        self._host = None
        return self

    def info(self):
        m, t, a, rx, ns = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        sc = C.c_double()
        _check(lib().chd_ct_info(self.ptr, C.byref(m), C.byref(t), C.byref(a), C.byref(rx),
                                 C.byref(sc), C.byref(ns)))
        return dict(num_main=m.value, num_ter=t.value, num_aux=a.value, has_rx=bool(rx.value),
                    scale=sc.value, num_slots=ns.value)

    def serialize(self):
        """The ciphertext as bytes (magic, shape, scale, slot count, primes,
        residues); Context.load_ct reads them back."""
        n = C.c_size_t()
        _check(lib().chd_ct_serialize(self.ctx.ptr, self.ptr, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().chd_ct_serialize(self.ctx.ptr, self.ptr, buf, n.value, C.byref(n)))
        return buf.raw

    def numpy(self):
        inf = self.info()
        rows = inf["num_main"] + inf["num_ter"] + inf["num_aux"]
        parts = [np.zeros((rows, self.ctx.n), dtype=np.uint32) for _ in range(3 if inf["has_rx"] else 2)]
        _check(lib().chd_ct_export(self.ctx.ptr, self.ptr, parts[0].ctypes.data, parts[1].ctypes.data,
                                   parts[2].ctypes.data if len(parts) > 2 else None, 0))
        return parts


class Client:
    """Test-only client on the device (the reference's UserInterface,
    src/UserInterface.cu): secrets, evaluation keys, encryption and
    decryption, reproducible from `seed`."""

    def __init__(self, ctx, seed):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        _check(lib().chd_client_create(ctx.ptr, seed, C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_client_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass

    def secret(self, sparse=False):
        rows = self.ctx.L + self.ctx.alpha
        out = np.zeros((rows, self.ctx.n), dtype=np.uint32)
        _check(lib().chd_client_secret(self.ctx.ptr, self.ptr, int(sparse), out.ctypes.data))
        return out

    def _key(self, fn, *args):
        k = EvaluationKey.__new__(EvaluationKey)
        k.ctx = self.ctx
        k.ptr = C.c_void_p()
        _check(fn(self.ctx.ptr, self.ptr, *args, C.byref(k.ptr)))
        return k

    def mult_key(self):
        return self._key(lib().chd_client_mult_key)

    def rotation_key(self, rot_idx):
        return self._key(lib().chd_client_rotation_key, rot_idx)

    def conjugation_key(self):
        return self._key(lib().chd_client_conjugation_key)

    def sse_keys(self):
        dts = EvaluationKey.__new__(EvaluationKey)
        std = EvaluationKey.__new__(EvaluationKey)
        dts.ctx = std.ctx = self.ctx
        dts.ptr, std.ptr = C.c_void_p(), C.c_void_p()
        _check(lib().chd_client_sse_keys(self.ctx.ptr, self.ptr, C.byref(dts.ptr), C.byref(std.ptr)))
        return dts, std

    def encrypt(self, pt, level, scale, num_slots=None, nonce=0):
        """pt: device plaintext (torch int32 [num_q(level)][N], as
        Context.encode returns it)."""
        ct = Ciphertext(self.ctx)
        _check(lib().chd_client_encrypt(self.ctx.ptr, self.ptr, nonce, level, scale,
                                        num_slots or self.ctx.n // 2, _ptr(pt), ct.ptr))
        return ct

    def decrypt(self, ct):
        import torch
        inf = ct.info()
        out = torch.empty((inf["num_main"] + inf["num_ter"], self.ctx.n), dtype=torch.int32, device="cuda")
        _check(lib().chd_client_decrypt(self.ctx.ptr, self.ptr, ct.ptr, _ptr(out)))
        return out

    def decrypt_decode(self, ct):
        """Decrypt, then decode with the ciphertext's level, scale and slot count."""
        inf = ct.info()
        level = self.ctx.level_of(inf["num_main"], inf["num_ter"])
        return self.ctx.decode(level, inf["scale"], self.decrypt(ct), inf["num_slots"])


class EvaluationKey:
    """EvaluationKey<uint32_t>: beta pairs over the key basis [L + alpha][N]."""

    def __init__(self, ctx, bx, ax, on_device=False, basis=None):
        """basis = (num_main, num_ter, num_aux) for a key over another basis
        than [L + alpha] (the dense-to-sparse key of sparse-secret
        encapsulation)."""
        self.ctx = ctx
        self.ptr = C.c_void_p()
        if on_device:
            beta = bx.shape[0]
            pb, pa = _ptr(bx), _ptr(ax)
        else:
            bx = np.ascontiguousarray(bx, dtype=np.uint32)
            ax = np.ascontiguousarray(ax, dtype=np.uint32)
            beta = bx.shape[0]
            pb, pa = bx.ctypes.data, ax.ctypes.data
        if basis is None:
            _check(lib().chd_evk_create(ctx.ptr, beta, pb, pa, int(on_device), C.byref(self.ptr)))
        else:
            _check(lib().chd_evk_create_np(ctx.ptr, basis[0], basis[1], basis[2], beta, pb, pa, int(on_device),
                                           C.byref(self.ptr)))

    def info(self):
        b, m, t, a = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().chd_evk_info(self.ptr, C.byref(b), C.byref(m), C.byref(t), C.byref(a)))
        return b.value, (m.value, t.value, a.value)

    def serialize(self):
        """The key as bytes; Context.load_evk reads them back."""
        n = C.c_size_t()
        _check(lib().chd_evk_serialize(self.ctx.ptr, self.ptr, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().chd_evk_serialize(self.ctx.ptr, self.ptr, buf, n.value, C.byref(n)))
        return buf.raw

    def numpy(self):
        """(bx, ax) as [beta][np][N] uint32 host arrays."""
        beta, (m, t, a) = self.info()
        bx = np.zeros((beta, m + t + a, self.ctx.n), dtype=np.uint32)
        ax = np.zeros_like(bx)
        _check(lib().chd_evk_export(self.ctx.ptr, self.ptr, bx.ctypes.data, ax.ctypes.data, 0))
        return bx, ax

    def __del__(self):
        try:
            if self.ptr.value:
                lib().chd_evk_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass


# ---------------------------------------------------------------- 64-bit words
class Context64:
    """The 64-bit word path (the reference's Context<uint64_t>): a context
    from a parameter JSON with primes up to 2^62 (e.g. the reference's
    bootparam_40_64bit.json), N = 2^16; raw NTT / ModUp / ModDown, HMult and
    HRot on uint64 residues."""

    def __init__(self, params_json, device=0):
        self.ptr = C.c_void_p()
        _check(lib().chd64_context_create_json(params_json.encode(), device, C.byref(self.ptr)))
        self.params = json.loads(params_json)
        self.n = 1 << self.params["log_degree"]
        self.max_level = lib().chd64_max_level(self.ptr)
        self.alpha = lib().chd64_alpha(self.ptr)

    def __del__(self):
        try:
            if getattr(self, "ptr", None) is not None and self.ptr.value:
                lib().chd64_context_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:  # interpreter teardown
            pass

    def synchronize(self):
        _check(lib().chd64_context_synchronize(self.ptr))

    def set_stream(self, stream_handle):
        """Run this context's work on the given CUDA stream (an int handle,
        e.g. torch.cuda.Stream().cuda_stream); None restores its own."""
        _check(lib().chd64_context_set_stream(self.ptr, stream_handle))

    def level_np(self, level):
        m, t = C.c_int(), C.c_int()
        _check(lib().chd64_level_np(self.ptr, level, C.byref(m), C.byref(t)))
        return m.value, t.value

    def scale(self, level):
        """Parameter::GetScale(level), up to the default encryption level."""
        return lib().chd64_scale(self.ptr, level)

    def primes(self):
        n = lib().chd64_primes(self.ptr, None, 0)
        out = np.zeros(n, dtype=np.uint64)
        lib().chd64_primes(self.ptr, out.ctypes.data, n)
        return out

    def ntt(self, np_, data_dev, count=1, inverse=False, mont=False):
        """NTT / INTT in place of `count` polynomials over (main, ter, aux)
        primes in a device tensor (int64 words)."""
        _check(lib().chd64_ntt(self.ptr, np_[0], np_[1], np_[2], _ptr(data_dev), count, int(inverse), int(mont)))

    def modup_raw(self, level, src_dev, dst_dev):
        _check(lib().chd64_modup_raw(self.ptr, level, _ptr(src_dev), _ptr(dst_dev)))

    def moddown_raw(self, level, kind, src_dev, dst_dev, npoly=1):
        _check(lib().chd64_moddown_raw(self.ptr, level, kind, _ptr(src_dev), _ptr(dst_dev), npoly))

    def import_ct(self, level, parts, scale=1.0, num_slots=None, on_device=False):
        return Ciphertext64(self).load(level, parts, scale, num_slots, on_device)

    def HMult(self, a, b, key, rescale=True, res=None):
        res = res or Ciphertext64(self)
        _check(lib().chd64_hmult(self.ptr, res.ptr, a.ptr, b.ptr, key.ptr, int(rescale)))
        return res

    def HRot(self, a, key, rot, res=None):
        res = res or Ciphertext64(self)
        _check(lib().chd64_hrot(self.ptr, res.ptr, a.ptr, key.ptr, rot))
        return res

    def HConj(self, a, key, res=None):
        res = res or Ciphertext64(self)
        _check(lib().chd64_hconj(self.ptr, res.ptr, a.ptr, key.ptr))
        return res

    def Rescale(self, a, res=None):
        res = res or Ciphertext64(self)
        _check(lib().chd64_rescale(self.ptr, res.ptr, a.ptr))
        return res

    # ---- Context<uint64_t> operations (Context.h:101-423) ----
    def _op(self, fn, res, *args):
        res = res or Ciphertext64(self)
        _check(fn(self.ptr, res.ptr, *args))
        return res

    def Copy(self, a, res=None):
        return self._op(lib().chd64_copy, res, a.ptr)

    def Neg(self, a, res=None):
        return self._op(lib().chd64_neg, res, a.ptr)

    def MultImaginaryUnit(self, a, res=None):
        return self._op(lib().chd64_mult_imaginary_unit, res, a.ptr)

    def Add(self, a, b, res=None):
        return self._op(lib().chd64_add, res, a.ptr, b.ptr)

    def Sub(self, a, b, res=None):
        return self._op(lib().chd64_sub, res, a.ptr, b.ptr)

    def Mult(self, a, b, res=None):
        """The three-part tensor (bx, ax, rx) of two ciphertexts."""
        return self._op(lib().chd64_mult, res, a.ptr, b.ptr)

    def Relinearize(self, a, key, res=None):
        return self._op(lib().chd64_relinearize, res, a.ptr, key.ptr, 0)

    def RelinearizeRescale(self, a, key, res=None):
        return self._op(lib().chd64_relinearize, res, a.ptr, key.ptr, 1)

    def MultKey(self, a, key, res=None):
        return self._op(lib().chd64_mult_key, res, a.ptr, key.ptr)

    def Permute(self, a, rot, res=None):
        return self._op(lib().chd64_permute, res, a.ptr, rot, 0)

    def PermuteConjugate(self, a, res=None):
        return self._op(lib().chd64_permute, res, a.ptr, 0, 1)

    def HRotAdd(self, a, b, key, rot, res=None):
        return self._op(lib().chd64_hrot_add, res, a.ptr, b.ptr, key.ptr, rot)

    def HConjAdd(self, a, b, key, res=None):
        return self._op(lib().chd64_hconj_add, res, a.ptr, b.ptr, key.ptr)

    def encode_const(self, level, scale, value, num_aux=0):
        """Encoder::EncodeConstant: one Montgomery word per prime."""
        m, t = self.level_np(level)
        out = np.zeros(m + t + num_aux, dtype=np.uint64)
        _check(lib().chd64_encode_const(self.ptr, level, float(scale), float(value), num_aux, out.ctypes.data))
        return out

    def MultConst(self, a, cx, const_scale, res=None):
        cx = np.ascontiguousarray(cx, dtype=np.uint64)
        return self._op(lib().chd64_mult_const, res, a.ptr, cx.ctypes.data, float(const_scale))

    def AddConst(self, a, cx, res=None):
        cx = np.ascontiguousarray(cx, dtype=np.uint64)
        return self._op(lib().chd64_add_const, res, a.ptr, cx.ctypes.data)

    def LevelDown(self, a, target_level, res=None):
        return self._op(lib().chd64_level_down, res, a.ptr, target_level)


class Ciphertext64:
    def __init__(self, ctx):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        _check(lib().chd64_ct_create(ctx.ptr, C.byref(self.ptr)))

    def __del__(self):
        try:
            if getattr(self, "ptr", None) is not None and self.ptr.value:
                lib().chd64_ct_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:  # interpreter teardown
            pass

    def load(self, level, parts, scale=1.0, num_slots=None, on_device=False):
        ns = self.ctx.n // 2 if num_slots is None else num_slots
        if on_device:
            ps = [_ptr(p) for p in parts]
            keep = parts
        else:
            keep = [np.ascontiguousarray(p, dtype=np.uint64) for p in parts]
            ps = [k.ctypes.data for k in keep]
        _check(lib().chd64_ct_import(self.ctx.ptr, self.ptr, level, scale, ns, ps[0], ps[1], int(on_device)))
        del keep
        return self

    def info(self):
        m, t, ns = C.c_int(), C.c_int(), C.c_int()
        sc = C.c_double()
        _check(lib().chd64_ct_info(self.ptr, C.byref(m), C.byref(t), C.byref(sc), C.byref(ns)))
        return dict(num_main=m.value, num_ter=t.value, scale=sc.value, num_slots=ns.value)

    def numpy(self):
        """(bx, ax), or (bx, ax, rx) for an unrelinearised ciphertext."""
        inf = self.info()
        rows = inf["num_main"] + inf["num_ter"]
        bx = np.zeros((rows, self.ctx.n), dtype=np.uint64)
        ax = np.zeros_like(bx)
        _check(lib().chd64_ct_export(self.ctx.ptr, self.ptr, bx.ctypes.data, ax.ctypes.data))
        if lib().chd64_ct_has_rx(self.ptr) == 1:
            rx = np.zeros_like(bx)
            _check(lib().chd64_ct_export_rx(self.ctx.ptr, self.ptr, rx.ctypes.data))
            return bx, ax, rx
        return bx, ax

    def set_rx(self, rx, on_device=False):
        keep = rx if on_device else np.ascontiguousarray(rx, dtype=np.uint64)
        _check(lib().chd64_ct_set_rx(self.ctx.ptr, self.ptr, _ptr(keep), int(on_device)))
        return self


class EvaluationKey64:
    """beta digits over the max-level key basis: bx, ax [beta][L + alpha][N]."""

    def __init__(self, ctx, bx, ax, on_device=False):
        self.ctx = ctx
        self.ptr = C.c_void_p()
        if on_device:
            beta, pb, pa, keep = bx.shape[0], _ptr(bx), _ptr(ax), None
        else:
            keep = (np.ascontiguousarray(bx, dtype=np.uint64), np.ascontiguousarray(ax, dtype=np.uint64))
            beta, pb, pa = keep[0].shape[0], keep[0].ctypes.data, keep[1].ctypes.data
        _check(lib().chd64_evk_create(ctx.ptr, beta, pb, pa, int(on_device), C.byref(self.ptr)))
        del keep

    def __del__(self):
        try:
            if getattr(self, "ptr", None) is not None and self.ptr.value:
                lib().chd64_evk_destroy(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:  # interpreter teardown
            pass
