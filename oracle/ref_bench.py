"""Times the reference's own evaluator (oracle/_ref/libcheddar_ref.so, the
reference's sources compiled for sm_100a) on the GPU, on the bench's
workloads, and prints one JSON line.  bench.py runs it as a separate process
(the reference keeps process-wide state per parameter set) after its own
measurements; the figures are the baseline the library is compared with,
not the library's.

    python oracle/ref_bench.py hmult <param file> <pairs> <steps> <warmup>
    python oracle/ref_bench.py ntt <primes> <polys> <steps> <warmup>
    python oracle/ref_bench.py boot <param file> <steps> <warmup>
    python oracle/ref_bench.py hmult64 <param file> <steps> <warmup>

Device time by CUDA events on the legacy stream the reference issues its
work on (the reference runs one ciphertext per call; it has no batched
entry points).  Inputs are resident on the device before timing starts.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
import refdrv  # noqa: E402

PARAMS = os.path.join(ROOT, "cheddar-fhe_b200", "params")


def _params(name):
    return json.load(open(os.path.join(PARAMS, name)))


def _uniform_ct(r, level, rng):
    m, t = r.level_np(level)
    q = r.prime_vector(m, t, 0).astype(np.uint64)[:, None]
    parts = [(rng.integers(0, 2 ** 62, size=(m + t, r.n), dtype=np.uint64) % q).astype(np.uint32)
             for _ in range(2)]
    return r.import_ct(m, t, 0, parts, r.test_scale(level), r.n // 2)


def hmult(name, pairs, steps, warmup):
    r = refdrv.RefContext(_params(name))
    lvl = r.max_level
    rng = np.random.default_rng(1)
    a = [_uniform_ct(r, lvl, rng) for _ in range(pairs)]
    b = [_uniform_ct(r, lvl, rng) for _ in range(pairs)]
    ms = r.time_hmult_set(a, b, steps, warmup=warmup)
    n = pairs * steps
    return {"workload": f"HMult+relin+rescale at the top level of {name}", "pairs_per_step": pairs,
            "steps": steps, "ms_per_hmult": ms / n, "hmult_per_s": n / (ms / 1e3)}


def ntt(nprimes, polys, steps, warmup):
    b = _params("bootparam_30.json")
    p = {"log_degree": 16, "log_default_scale": 30, "boot": False, "dense_hamming_weight": 192,
         "sparse_hamming_weight": 32, "terminal_primes": [], "main_primes": b["main_primes"][2:2 + nprimes],
         "auxiliary_primes": b["auxiliary_primes"][:8], "default_encryption_level": nprimes - 1,
         "level_config": [[i, 0] for i in range(1, nprimes + 1)], "additional_base": [0, 0]}
    r = refdrv.RefContext(p)
    ms = r.time_ntt_roundtrip(nprimes, polys, steps, warmup=warmup)
    n = polys * steps
    return {"workload": f"NTT + INTT round trip, {nprimes} primes main_primes[2..{nprimes + 1}] of "
                        "bootparam_30.json", "polys_per_step": polys, "steps": steps,
            "us_per_roundtrip": 1e3 * ms / n}


def boot(name, steps, warmup):
    p = _params(name)
    r = refdrv.RefContext(p)
    rots = r.boot_prepare(r.n // 2)
    rng = np.random.default_rng(3)
    msg = (rng.random(r.n // 2) * 2 - 1) + 1j * (rng.random(r.n // 2) * 2 - 1)
    c = r.encrypt(0, msg)
    out = {"workload": f"full-slot Boot of {name}", "rotation_keys": len(rots), "steps": steps}
    for min_ks in (False, True):
        ms = r.time_boot(c, steps, warmup=warmup, min_ks=min_ks)
        out["min_ks" if min_ks else "hoisted"] = {"ms_per_boot": ms / steps, "bootstraps_per_s": steps / (ms / 1e3)}
    return out


def w64_inputs(p, seed=1):
    """Uniform level-max ciphertext pair and key of the 64-bit word path
    (the same residues for the reference and the library)."""
    n = 1 << p["log_degree"]
    primes = list(reversed(p.get("terminal_primes", []))) + p["main_primes"] + p["auxiliary_primes"]
    na, L = len(p["auxiliary_primes"]), len(p["main_primes"]) + len(p.get("terminal_primes", []))
    rng = np.random.default_rng(seed)

    def uni(rows):
        return np.stack([rng.integers(0, primes[r], n, dtype=np.uint64) for r in rows])
    beta = -(-L // na)
    key = (np.stack([uni(range(L + na)) for _ in range(beta)]), np.stack([uni(range(L + na)) for _ in range(beta)]))
    a = (uni(range(L)), uni(range(L)))
    b = (uni(range(L)), uni(range(L)))
    return a, b, key


def hmult64(name, steps, warmup):
    p = _params(name)
    r = refdrv.RefContext64(p)
    a, b, key = w64_inputs(p)
    lvl = len(p["level_config"]) - 1
    ms = r.time_hmult(lvl, a, b, key, True, warmup, steps)
    return {"workload": f"64-bit word path: HMult+relin+rescale at the top level of {name}", "steps": steps,
            "ms_per_hmult": ms, "hmult_per_s": 1e3 / ms}


def main(argv):
    kind = argv[1]
    if kind == "hmult":
        res = hmult(argv[2], int(argv[3]), int(argv[4]), int(argv[5]))
    elif kind == "ntt":
        res = ntt(int(argv[2]), int(argv[3]), int(argv[4]), int(argv[5]))
    elif kind == "boot":
        res = boot(argv[2], int(argv[3]), int(argv[4]))
    elif kind == "hmult64":
        res = hmult64(argv[2], int(argv[3]), int(argv[4]))
    else:
        raise SystemExit(f"unknown workload {kind}")
    print(json.dumps({"reference_gpu": kind, **res}), flush=True)
    os._exit(0)


if __name__ == "__main__":
    main(sys.argv)
