"""Parity pinned to the reference's own evaluator.

The reference's library (its src/core, src/extension and
src/UserInterface.cu, compiled for sm_100a from its own sources by
`make -C oracle ref`, with project-written stand-ins for rmm and libtommath)
runs beside this library and the CPU oracle on identical inputs and on the
reference's own keys and encryptions; every residue must be equal:

* ntt24: NTT / INTT over main_primes[2..25] of bootparam_30.json;
* modswitch: ModUp, ModDown, Rescale, ModDownAndRescale;
* keyswitch: HMult (with and without rescale), HRot, HConj, Rescale;
* hoisted: 30 hoisted baby-step rotations (EvaluateBabyStep);
* context_ops, context_ops40: Add, Sub, Neg, Mult, Relinearize(Rescale),
  Rescale, MultKey, Permute, MultImaginaryUnit, LevelDown, HRotAdd,
  HConjAdd, MultUnsafe, HMult, on the L = 24 set and on bootparam_40.json
  (terminal primes, rational rescale);
* encode, decode: the encoder at several levels, scales and aux counts; the
  decoder, double for double, on the reference's decryptions;
* boot40, boot30, boot35: full-slot Boot, hoisted and min-KS, and
  BootBatch, on the reference's bootparam_{40,30,35}.json exactly, with the
  reference's decoded precision; boot40_sparse: 2^10 slots.

Each case runs in its own process (tests/refpin_cases.py explains why).
"""
import json
import os
import subprocess
import sys

import pytest

import conftest
import refdrv

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("case", ["ntt24", "modswitch", "keyswitch", "mixed_batch", "w64", "w64_ops", "hoisted", "context_ops", "context_ops40",
                                  "encode", "decode", "boot40", "boot30", "boot35", "boot40_sparse"])
def test_reference_parity(cuda_ok, case):
    if not refdrv.available():
        pytest.fail("oracle/_ref/libcheddar_ref.so is missing: build it with `make -C oracle ref REF=<tree>`")
    r = subprocess.run([sys.executable, os.path.join(HERE, "refpin_cases.py"), case], capture_output=True,
                       text=True, timeout=1500)
    sys.stdout.write(r.stdout)
    sys.stderr.write(r.stderr[-4000:])
    assert r.returncode == 0, f"case {case} failed (rc {r.returncode}):\n{r.stderr[-3000:]}"
    line = [x for x in r.stdout.splitlines() if x.startswith("{")][-1]
    assert json.loads(line)["case"] == case
    conftest.REPORT.append(line)
