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

PARAMS = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "..", "cheddar-fhe_b200", "params", "*.json")))


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
