"""Decoded precision of one full-slot bootstrap at N = 2^16 with real keys.

Not collected by pytest (key generation by the oracle at this size takes a
few minutes); run it on a GPU machine as

    python tests/boot_precision_n16.py [parameter file]

The oracle generates the secret, every evaluation key (with the
dense-to-sparse and sparse-to-dense keys when the parameters use
sparse-secret encapsulation), encrypts uniform slots in [-1, 1]^2 at level 0
and decodes the library's bootstrap; the script prints the precision in bits
(-log2 of the largest slot error) as one JSON line.  The oracle is the
checker here: the bootstrap itself runs in the CUDA library.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "cheddar-fhe_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cheddar_b200 as chd  # noqa: E402
import pyoracle as po  # noqa: E402
from boot_oracle import gen_sse_keys  # noqa: E402


def main(name="boot40_l28_a12.json"):
    params = json.load(open(os.path.join(chd.PARAM_DIR, name)))
    ctx = chd.Context(json.dumps(params))
    bc = chd.BootContext(ctx)
    o = po.Oracle(params)
    sse = params["dense_hamming_weight"] != params["sparse_hamming_weight"]
    s = o.gen_secret(99, params["dense_hamming_weight"] if sse else params["sparse_hamming_weight"])
    keys = chd.EvkMap(ctx)
    held = [ctx.evk(*o.gen_mult_key(77, s)), ctx.evk(*o.gen_conj_key(78, s))]
    keys.set_mult(held[0])
    keys.set_conjugation(held[1])
    for r in bc.rotations():
        held.append(ctx.evk(*o.gen_rot_key(1000 + r, s, r)))
        keys.set_rotation(r, held[-1])
    if sse:
        dts, std = gen_sse_keys(o, 377, s, o.gen_secret(299, params["sparse_hamming_weight"]))
        m, t = o.level_np(-1)
        held.append(chd.EvaluationKey(ctx, dts[0], dts[1], basis=(m, t, m + t)))
        keys.set_dense_to_sparse(held[-1])
        held.append(chd.EvaluationKey(ctx, std[0], std[1], basis=(o.L - o.max_ter, o.max_ter, o.alpha)))
        keys.set_sparse_to_dense(held[-1])
    rng = np.random.default_rng(2024)
    msg = (rng.random(o.n // 2) * 2 - 1) + 1j * (rng.random(o.n // 2) * 2 - 1)
    bx, ax = o.encrypt(5, s, 0, o.encode(0, o.scale(0), msg))
    r = bc.Boot(ctx.import_ct(0, [bx, ax], o.scale(0)), keys)
    dec = o.decode(bc.end_level, bc.final_scale, o.decrypt(s, bc.end_level, r.numpy()), o.n // 2)
    err = float(np.abs(dec - msg).max())
    print(json.dumps({"params": name, "n": o.n, "slots": o.n // 2, "bits": -float(np.log2(err)),
                      "max_abs_error": err, "encapsulation": sse}))


if __name__ == "__main__":
    main(*sys.argv[1:])
