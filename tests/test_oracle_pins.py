"""Pins of the CPU oracle against the reference's own code.

* primeutil_ref.jsonl was produced by the reference's include/common/
  PrimeUtils.h (+ Normalize, BitReverseVector) compiled from the reference
  tree (tests/golden/make_golden.py).  The oracle's restatement must agree on
  every prime.
* basic_pin (GPU) runs the reference's Basic.cuh Montgomery primitives for
  sm_100a and the oracle must reproduce every output word, including the
  lazy (-q, q) results.
"""
import json
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "primeutil_ref.jsonl")


def _fnv(words):
    h = 1469598103934665603
    b = np.asarray(words, dtype="<u4").tobytes()
    for x in b:
        h ^= x
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


def _records():
    with open(GOLDEN) as f:
        return [json.loads(l) for l in f if l.strip()]


def test_golden_prime_utils():
    L = po.lib()
    recs = _records()
    assert len(recs) >= 50
    for r in recs:
        p = r["prime"]
        assert L.orc_find_generator(p) == r["generator"], p
        psi = L.orc_primitive_root(1 << 17, p)
        assert psi == r["psi"], p
        assert L.orc_inv_mod(psi, p) == r["psi_inv"], p
        assert L.orc_inv_mod_base(p) == r["q_inv"], p
        assert L.orc_inv_mod(1 << 16, p) == r["n_inv"], p
        assert L.orc_to_mont(L.orc_to_mont(1, p), p) == r["r2"], p
        assert L.orc_normalize(p - 1, p) == r["normalize_hi"]
        assert L.orc_normalize(p >> 1, p) == r["normalize_mid"]
        assert L.orc_pow_mod(12345, -77, p) == r["pow_neg"]


def test_golden_twiddle_tables():
    """The oracle's bit-reversed Montgomery twiddle tables hash-equal the
    tables built by the reference's PrimeUtils (all primes of the
    key-switching parameter set)."""
    o = po.Oracle(po.load_param_json(
        os.path.join(os.path.dirname(__file__), "..", "cheddar-fhe_b200", "params", "keyswitch_l24_a8.json")))
    by_p = {r["prime"]: r for r in _records()}
    primes = o.all_primes()
    for g, p in enumerate(primes):
        tw, itw = o.twiddles(g)
        r = by_p[int(p)]
        assert list(tw[:4]) == r["tw_head"]
        assert _fnv(tw) == r["tw_hash"], p
        assert _fnv(itw) == r["itw_hash"], p


@pytest.mark.gpu
def test_reference_basic_cuh_on_gpu(cuda_ok):
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "basic_pin")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/basic_pin not built (needs the reference tree)")
    primes = [786433, 33292289, 1073479681, 2130444289, 2147352577]
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "pin.bin")
        subprocess.run([exe, out] + [str(p) for p in primes], check=True, timeout=120)
        raw = open(out, "rb").read()
    cnt = struct.unpack_from("<I", raw, 0)[0]
    rec = np.frombuffer(raw, dtype=np.dtype([("q", "<u4"), ("qinv", "<i4"), ("a", "<i4"), ("b", "<i4"),
                                               ("lazy", "<i4"), ("mont", "<u4"), ("red", "<u4"),
                                               ("norm", "<i4")]), count=cnt, offset=4)
    L = po.lib()
    for x in rec[:: max(1, cnt // 4000)]:
        q, qi, a, b = int(x["q"]), int(x["qinv"]), int(x["a"]), int(x["b"])
        assert L.orc_mont_mult_lazy(a, b, q, qi) == int(x["lazy"])
        ua, ub = (a + q if a < 0 else a), (b + q if b < 0 else b)
        assert L.orc_mont_mult(ua, ub, q, qi) == int(x["mont"])
        assert L.orc_mont_reduce(a * b, q, qi) == int(x["red"])
        assert L.orc_normalize(ua, q) == int(x["norm"])
