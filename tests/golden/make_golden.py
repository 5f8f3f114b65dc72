"""Regenerate the golden fixtures pinned on the reference's own sources.

primeutil_ref.jsonl: output of oracle/_ref/primeutil_pin, a driver compiled
(by `make -C oracle ref`) from the reference tree's include/common/
PrimeUtils.h, Basic.cuh (Normalize) and CommonUtils.h (BitReverseVector).
For every prime of the parameter files used by the tests and benchmarks it
records the generator, psi, psi^-1, q^-1 mod 2^32, N^-1, R^2 mod q and
hashes of the bit-reversed Montgomery twiddle tables, computed by the
reference's code.  The oracle is checked against this file in
tests/test_oracle_pins.py.

Run from the repository root (needs the reference tree; no GPU):
    CHEDDAR_REFERENCE=<reference tree> python tests/golden/make_golden.py
"""
import glob
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    tree = os.environ.get("CHEDDAR_REFERENCE")
    if not tree:
        raise SystemExit("set CHEDDAR_REFERENCE to the reference source tree")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={tree}"], check=True)
    primes = set()
    for f in sorted(glob.glob(os.path.join(ROOT, "cheddar-fhe_b200", "params", "*.json"))):
        d = json.load(open(f))
        for k in ("main_primes", "auxiliary_primes", "terminal_primes"):
            primes.update(d.get(k, []))
    primes = sorted(primes)
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "primeutil_pin"), "16"] + [str(p) for p in primes],
                         check=True, capture_output=True, text=True).stdout
    path = os.path.join(ROOT, "tests", "golden", "primeutil_ref.jsonl")
    with open(path, "w") as f:
        f.write(out)
    print(f"wrote {path}: {len(primes)} primes")


if __name__ == "__main__":
    sys.exit(main())
