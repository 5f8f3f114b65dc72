"""The parameter files shipped with the library are exactly what
cheddar-fhe_b200/params/gen_params.py generates, and every prime in them is
distinct, below 2^31, prime and NTT-friendly for N = 2^16 (p = 1 mod 2^17),
as Parameter.cu:40-62 of the reference requires (no GPU needed)."""
import importlib.util
import json
import os

import pytest

PARAMS = os.path.join(os.path.dirname(__file__), "..", "cheddar-fhe_b200", "params")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_params", os.path.join(PARAMS, "gen_params.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


GEN = _gen()
FILES = {
    "keyswitch_l24_a8.json": lambda: GEN.keyswitch_params(24, 8),
    "keyswitch_l8_a3.json": lambda: GEN.keyswitch_params(8, 3),
    "rational_t4_m10_a6.json": GEN.rational_params,
    "boot_l34_a12.json": GEN.boot_params,
    "boot_l34_a12_sse.json": lambda: dict(GEN.boot_params(), dense_hamming_weight=32768),
    "boot40_l28_a12.json": GEN.boot40_params,
    "ntt_bootparam30_p24.json": GEN.ntt_bootparam30_params,
}
# the reference's own parameter sets, shipped unchanged
REFERENCE_FILES = ["bootparam_30.json", "bootparam_35.json", "bootparam_40.json"]


@pytest.mark.parametrize("name", sorted(FILES))
def test_file_is_generated(name):
    assert json.load(open(os.path.join(PARAMS, name))) == FILES[name]()


@pytest.mark.parametrize("name", sorted(FILES))
def test_primes_valid(name):
    p = json.load(open(os.path.join(PARAMS, name)))
    primes = p["terminal_primes"] + p["main_primes"] + p["auxiliary_primes"]
    assert len(set(primes)) == len(primes)
    for q in primes:
        assert q < (1 << 31) and q % (1 << 17) == 1 and GEN.is_prime(q)
    assert len(primes) <= 64
    # every level holds at most the primes the set has, and the top level all of them
    main, ter = len(p["main_primes"]), len(p["terminal_primes"])
    assert all(0 <= m <= main and 0 <= t <= ter for m, t in p["level_config"])
    assert p["level_config"][-1] == [main, ter]


def test_boot40_shape():
    p = json.load(open(os.path.join(PARAMS, "boot40_l28_a12.json")))
    assert (len(p["terminal_primes"]), len(p["main_primes"]), len(p["auxiliary_primes"])) == (4, 43, 12)
    assert len(p["level_config"]) == 29 and p["default_encryption_level"] == 16
    assert p["log_default_scale"] == 40 and p["dense_hamming_weight"] != p["sparse_hamming_weight"]


# sha256 of the reference's parameter files (parameters/bootparam_*.json of
# scale-snu/cheddar-fhe), which ship here unchanged
REFERENCE_SHA256 = {
    "bootparam_30.json": "17d0b20eeb75759598146222e9734aee6bdd2cc42d27eba441e9fdd6b57cf787",
    "bootparam_35.json": "402f088aeb29dfb1908760f5d072e1c9f03713a83dbca5e793f58fe99fc7a9ad",
    "bootparam_40.json": "a54027c59166d3e28c02fd619d9e7eea4fc2b14524b32c789aee60b114686e2e",
    "bootparam_40_64bit.json": "1b9f9b635e82eb4e67344a22fe466b7f9a6764075a3e9ca2ff1e053e3a3678dd",
}


@pytest.mark.parametrize("name", REFERENCE_FILES)
def test_reference_parameter_files(name):
    import hashlib
    path = os.path.join(PARAMS, name)
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == REFERENCE_SHA256[name]
    p = json.load(open(path))
    primes = p["terminal_primes"] + p["main_primes"] + p["auxiliary_primes"]
    assert len(set(primes)) == len(primes) and len(primes) <= 64
    for q in primes:
        assert q < (1 << 31) and q % (1 << 17) == 1 and GEN.is_prime(q)
    main, ter = len(p["main_primes"]), len(p["terminal_primes"])
    assert p["level_config"][-1] == [main, ter]


def test_bootparam40_shape():
    p = json.load(open(os.path.join(PARAMS, "bootparam_40.json")))
    assert (len(p["terminal_primes"]), len(p["main_primes"]), len(p["auxiliary_primes"])) == (4, 43, 12)
    assert (p["num_cts_levels"], p["num_stc_levels"], p["default_encryption_level"]) == (4, 3, 16)


def _is_prime64(n):
    # deterministic Miller-Rabin for n < 3.3e24
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def test_reference_64bit_parameter_file():
    # the reference's parameter set of its 64-bit word path, unchanged:
    # 40-55-bit main primes, 56-bit auxiliary primes, all below the 2^62 the
    # 64-bit path accepts, NTT-friendly for N = 2^16, exact as JSON integers
    import hashlib
    name = "bootparam_40_64bit.json"
    path = os.path.join(PARAMS, name)
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == REFERENCE_SHA256[name]
    p = json.load(open(path))
    primes = p["terminal_primes"] + p["main_primes"] + p["auxiliary_primes"]
    assert len(set(primes)) == len(primes) and len(primes) <= 64
    assert max(primes) >= (1 << 53)  # beyond a double: the parser must read integers exactly
    for q in primes:
        assert q < (1 << 62) and q % (1 << 17) == 1 and _is_prime64(q)
    assert p["level_config"][-1] == [len(p["main_primes"]), len(p["terminal_primes"])]
