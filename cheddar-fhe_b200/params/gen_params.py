"""Generate CKKS parameter files in the reference's JSON schema.

The schema (log_degree, log_default_scale, default_encryption_level,
main_primes, terminal_primes, auxiliary_primes, level_config,
additional_base, dense/sparse_hamming_weight, boot, num_cts_levels,
num_stc_levels) is the one the reference's test bed parses
(unittest/Testbed.h:95-221 of scale-snu/cheddar-fhe).  The primes are found
here: NTT-friendly (p = 1 mod 2N for N = 2^16, hence for every smaller N)
and below 2^31, as Parameter.cu:40-62 requires.

Run:  python gen_params.py   (rewrites the *.json files beside this script)
"""
import json
import os

TWO_N = 1 << 17


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17):  # deterministic below 3.4e14
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


def primes_near(target, count, used, direction):
    """`count` primes p = 1 mod 2^17 walking away from `target`."""
    out = []
    k = target // TWO_N
    while len(out) < count:
        p = k * TWO_N + 1
        if p < (1 << 31) and p not in used and is_prime(p):
            out.append(p)
            used.add(p)
        k += direction
    return out


def alternating(target, count, used):
    """Primes alternately just above and just below `target` so that the
    running product of rescaled primes stays close to target^k."""
    up = primes_near(target, (count + 1) // 2, used, +1)
    down = primes_near(target, count // 2, used, -1)
    out = []
    for i in range(count):
        out.append(up[i // 2] if i % 2 == 0 else down[i // 2])
    return out


def keyswitch_params(num_main, num_aux, log_n=16, log_scale=30):
    used = set()
    aux = primes_near((1 << 31) - 1, num_aux, used, -1)
    main = alternating(1 << log_scale, num_main, used)
    levels = [[k, 0] for k in range(2, num_main + 1)]
    return {
        "log_degree": log_n,
        "log_default_scale": log_scale,
        "boot": False,
        "dense_hamming_weight": 192,
        "sparse_hamming_weight": 32,
        "terminal_primes": [],
        "main_primes": main,
        "auxiliary_primes": aux,
        "default_encryption_level": len(levels) - 1,
        "level_config": levels,
        "additional_base": [0, 0],
    }


def rational_params(log_n=16):
    """A small parameter set with terminal primes and rational rescale
    (levels that drop main primes while restoring terminal primes and vice
    versa), for exercising the restore/padding constants of the merged
    ModDown+Rescale."""
    used = set()
    aux = primes_near((1 << 31) - 1, 6, used, -1)
    ter = primes_near(1 << 25, 4, used, +1)
    main = alternating(1 << 30, 10, used)
    levels = [[0, 2], [3, 0], [1, 4], [4, 2], [7, 0], [5, 4], [8, 2],
              [10, 0], [10, 2], [10, 4]]
    return {
        "log_degree": log_n,
        "log_default_scale": 30,
        "boot": False,
        "dense_hamming_weight": 192,
        "sparse_hamming_weight": 32,
        "terminal_primes": ter,
        "main_primes": main,
        "auxiliary_primes": aux,
        "default_encryption_level": 7,
        "level_config": levels,
        "additional_base": [0, 0],
    }


def boot_params(log_n=16):
    """The shape of the reference's bootparam_30.json: two ~20-bit base
    primes (level 0 and the level -1 base), 22 primes near 2^30 (one per
    level), then 12 levels of two primes near 2^29 each (the CoeffToSlot
    and EvalMod levels), 12 auxiliary primes; 4 CtS and 3 StC levels.  The
    secret is sparse (Hamming weight 32) and sparse-secret encapsulation is
    off (dense = sparse weight)."""
    used = set()
    aux = primes_near((1 << 31) - 1, 12, used, -1)
    base = primes_near(1 << 20, 2, used, +1)
    mid = alternating(1 << 30, 22, used)
    top = alternating(1 << 29, 24, used)
    levels = [[k, 0] for k in range(2, 25)] + [[k, 0] for k in range(26, 49, 2)]
    return {
        "log_degree": log_n,
        "log_default_scale": 30,
        "boot": True,
        "dense_hamming_weight": 32,
        "sparse_hamming_weight": 32,
        "num_cts_levels": 4,
        "num_stc_levels": 3,
        "terminal_primes": [],
        "main_primes": base + mid + top,
        "auxiliary_primes": aux,
        "default_encryption_level": 22,
        "level_config": levels,
        "additional_base": [0, 0],
    }


def boot40_params(log_n=16):
    """The shape of the reference's bootparam_40.json (40-bit scale from
    32-bit words by rational rescale): 4 terminal primes near 2^25, 23 main
    primes near 2^30 for the levels that mix main and terminal primes, 16
    near 2^29 for the two-prime bootstrapping levels, 4 more near 2^30, and
    12 auxiliary primes; its level table (the primes each level holds, a
    property of the workload, kept as the reference defines it); 4 CtS and 3
    StC levels; sparse-secret encapsulation on (dense Hamming weight 32768,
    sparse 32).  The primes are this generator's own."""
    used = set()
    aux = primes_near((1 << 31) - 1, 12, used, -1)
    ter = primes_near(1 << 25, 4, used, +1)
    main = alternating(1 << 30, 23, used) + alternating(1 << 29, 16, used) + alternating(1 << 30, 4, used)
    levels = [[0, 2], [3, 0], [1, 4], [4, 2], [7, 0], [5, 4], [8, 2], [11, 0], [9, 4], [12, 2], [15, 0],
              [13, 4], [16, 2], [19, 0], [17, 4], [20, 2]] + [[k, 0] for k in range(23, 44, 2)] + [[43, 2], [43, 4]]
    return {
        "log_degree": log_n,
        "log_default_scale": 40,
        "boot": True,
        "dense_hamming_weight": 32768,
        "sparse_hamming_weight": 32,
        "num_cts_levels": 4,
        "num_stc_levels": 3,
        "terminal_primes": ter,
        "main_primes": main,
        "auxiliary_primes": aux,
        "default_encryption_level": 16,
        "level_config": levels,
        "additional_base": [0, 0],
    }


def ntt_bootparam30_params():
    """The NTT workload's primes: main_primes[2..25] of the reference's own
    bootparam_30.json (shipped beside this script), the 24 primes near 2^30
    that follow its two ~20-bit base primes, as the q basis of a 24-level
    chain (one prime per level), with that file's first 8 auxiliary
    primes."""
    here = os.path.dirname(os.path.abspath(__file__))
    ref = json.load(open(os.path.join(here, "bootparam_30.json")))
    return {
        "log_degree": 16,
        "log_default_scale": 30,
        "boot": False,
        "dense_hamming_weight": 192,
        "sparse_hamming_weight": 32,
        "terminal_primes": [],
        "main_primes": ref["main_primes"][2:26],
        "auxiliary_primes": ref["auxiliary_primes"][:8],
        "default_encryption_level": 23,
        "level_config": [[i, 0] for i in range(1, 25)],
        "additional_base": [0, 0],
    }


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    files = {
        # L = 24 q primes + alpha = 8 aux primes: dnum = 3 at the top level
        "keyswitch_l24_a8.json": keyswitch_params(24, 8),
        # small: L = 8 + alpha = 3 (beta = 3, ragged last digit)
        "keyswitch_l8_a3.json": keyswitch_params(8, 3),
        "rational_t4_m10_a6.json": rational_params(),
        # bootstrapping: 48 q primes (max level 34) + alpha = 12 aux primes
        "boot_l34_a12.json": boot_params(),
        # the same with sparse-secret encapsulation (dense Hamming weight
        # 32768 > sparse 32), as the reference's bootparam_*.json files
        "boot_l34_a12_sse.json": dict(boot_params(), dense_hamming_weight=32768),
        # bootstrapping with the reference's 40-bit parameter shape: 4
        # terminal + 43 main primes (max level 28), alpha = 12
        "boot40_l28_a12.json": boot40_params(),
        # the NTT workload on the reference's own primes
        "ntt_bootparam30_p24.json": ntt_bootparam30_params(),
    }
    for name, obj in files.items():
        with open(os.path.join(here, name), "w") as f:
            json.dump(obj, f, indent=1)
            f.write("\n")
        print("wrote", name)


if __name__ == "__main__":
    main()
