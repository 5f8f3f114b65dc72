"""The CUDA library's host-side ModSwitch constants (computed without a GPU
by chd_params_level_consts) equal the oracle's restatement of the
reference's ModSwitchHandler constructor (src/core/ModSwitch.cu:175-411) for
every level, digit and ModDown variant of every parameter set."""
import ctypes as C
import glob
import json
import os

import numpy as np
import pytest

import cheddar_b200 as chd
import pyoracle as po

# 32-bit word parameter sets (the 64-bit word path has its own parity case)
PARAMS = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "..", "cheddar-fhe_b200", "params",
                                                  "*.json")) if not p.endswith("_64bit.json"))


@pytest.mark.parametrize("path", PARAMS, ids=[os.path.basename(p) for p in PARAMS])
def test_level_constants_match_oracle(path):
    p = json.load(open(path))
    p["log_degree"] = 12
    o = po.Oracle(p)
    js = json.dumps(p).encode()
    L, OL = chd.lib(), po.lib()
    L.chd_params_level_consts.restype = C.c_int
    OL.orc_level_consts.restype = C.c_int
    checked = 0
    for lvl in range(-1, o.max_level + 1):
        for kind in range(4):
            for d in (range(o.beta(lvl)) if kind == 0 else [0]):
                a = [np.zeros(64, np.uint32), np.zeros(64 * 16, np.int32), np.zeros(64, np.uint32),
                     np.zeros(64, np.uint32), np.zeros(6, np.int32)]
                b = [np.zeros_like(x) for x in a]
                r1 = L.chd_params_level_consts(js, lvl, kind, d, *[x.ctypes.data_as(C.c_void_p) for x in a])
                r2 = OL.orc_level_consts(C.c_void_p(o.ptr), lvl, kind, d, *[x.ctypes.data_as(C.c_void_p) for x in b])
                assert (r1 == 0) == (r2 == 0), (lvl, kind, d)
                if r1 == 0:
                    for x, y in zip(a, b):
                        assert np.array_equal(x, y), (lvl, kind, d)
                    checked += 1
    assert checked > o.max_level


def test_more_than_64_primes_rejected():
    # the extended basis lives in 64-entry tables: a parameter set with more
    # primes is refused when parsed (no GPU needed), not overrun later
    p = json.load(open(PARAMS[0]))
    p["log_degree"] = 12
    step = 2 << 12
    p["main_primes"] = [1 + step * k for k in range(1, 58)]
    p["terminal_primes"] = []
    p["auxiliary_primes"] = [1 + step * k for k in range(100, 108)]
    p["level_config"] = [[k, 0] for k in range(2, 58)]
    L = chd.lib()
    L.chd_params_level_consts.restype = C.c_int
    a = [np.zeros(64, np.uint32), np.zeros(64 * 16, np.int32), np.zeros(64, np.uint32),
         np.zeros(64, np.uint32), np.zeros(6, np.int32)]
    rc = L.chd_params_level_consts(json.dumps(p).encode(), 0, 0, 0, *[x.ctypes.data_as(C.c_void_p) for x in a])
    assert rc != 0
    assert b"64" in L.chd_last_error()
