"""CPU checks of the C ABI library: it loads without a GPU, exports every
entry point include/cheddar_b200.h declares, and its host-side parameter
validation reports errors (no GPU call is made on these paths)."""
import ctypes as C
import json
import os
import re

import pytest

import cheddar_b200 as chd

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "cheddar_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 40
    for s in ("chd_hmult", "chd_hrot", "chd_hoisted_rotate", "chd_ntt", "chd_bconv_raw",
              "chd_context_create_json", "chd_moddown_raw"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(chd.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_json_parse_error_is_reported():
    L = chd.lib()
    out = C.c_void_p()
    rc = L.chd_context_create_json(b"{ not json", 0, C.byref(out))
    assert rc == 8  # CHD_ERR_PARSE
    assert "JSON" in L.chd_last_error().decode()


def test_missing_field_is_reported():
    L = chd.lib()
    out = C.c_void_p()
    rc = L.chd_context_create_json(json.dumps({"log_degree": 16}).encode(), 0, C.byref(out))
    assert rc == 8
    assert "Missing" in L.chd_last_error().decode()


@pytest.mark.parametrize("bad, msg", [
    ({"main_primes": [1073872897, 12289]}, "NTT-friendly"),
    ({"level_config": [[2, 0], [1, 0], [24, 0]]}, "level configuration"),
    ({"auxiliary_primes": [4294967291]}, "too large"),
])
def test_invalid_parameters_are_rejected(bad, msg):
    p = json.load(open(os.path.join(chd.PARAM_DIR, "keyswitch_l24_a8.json")))
    p.update(bad)
    L = chd.lib()
    out = C.c_void_p()
    rc = L.chd_context_create_json(json.dumps(p).encode(), 0, C.byref(out))
    assert rc != 0
    assert msg in L.chd_last_error().decode()


def test_null_arguments_are_rejected():
    L = chd.lib()
    assert L.chd_hmult(None, None, None, None, None, 1) == 1
    assert "null" in L.chd_last_error().decode()
