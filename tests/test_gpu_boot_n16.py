"""Batched bootstrapping at the full size (N = 2^16, 2^15 slots; the
bootstrapping parameter sets with 48 q primes, and with the reference's
40-bit shape of 4 terminal + 43 main primes, alpha = 12): BootBatch of
three ciphertexts equals Boot of each, bit for bit, with the hoisted and
with the min-KS linear transforms.  At N = 2^16 every key switch runs the
fused pipeline (column passes, key-switch row pass) and the batched kernels
(giant-step accumulation over the batch, hoisted rotations of the batch,
giant-step key switches kept in Q u P), which the N = 2^12 bootstrapping
tests do not reach.  Keys and inputs are uniform random residues: the
residue arithmetic, not decryption, is under test (decoded precision at this
size is measured by tests/boot_precision_n16.py)."""
import functools
import json
import os

import numpy as np
import pytest

import cheddar_b200 as chd

pytestmark = pytest.mark.gpu
BOOTS = ["boot_l34_a12.json", "boot40_l28_a12.json"]
B = 3


@functools.lru_cache(maxsize=None)
def _setup(name):
    import torch
    params = json.load(open(os.path.join(chd.PARAM_DIR, name)))
    ctx = chd.Context(json.dumps(params))
    bc = chd.BootContext(ctx)
    rots = sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True)))
    n, L, a = ctx.n, ctx.L, ctx.alpha
    beta = -(-L // a)
    allp = torch.tensor(list(reversed(params.get("terminal_primes", []))) + params["main_primes"] +
                        params["auxiliary_primes"], dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(2024)

    def uniform(rows_gidx):
        q = allp[torch.tensor(rows_gidx, device="cuda", dtype=torch.int64)][:, None]
        r = torch.randint(0, 2 ** 62, (len(rows_gidx), n), generator=gen, device="cuda", dtype=torch.int64)
        return (r % q).to(torch.int32)

    kg = list(ctx.gidx(*ctx.level_np(ctx.max_level), a))
    keys = chd.EvkMap(ctx)
    held = []

    def ukey():
        kb = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        ka = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        k = chd.EvaluationKey(ctx, kb, ka, on_device=True)
        held.append(k)
        return k

    keys.set_mult(ukey())
    keys.set_conjugation(ukey())
    for r in rots:
        keys.set_rotation(r, ukey())
    if params["dense_hamming_weight"] != params["sparse_hamming_weight"]:
        # sparse-secret encapsulation: the dense-to-sparse key over the level
        # -1 primes and as many auxiliary primes, the sparse-to-dense key as
        # one digit over the whole key basis
        m, t = ctx.level_np(-1)
        g_dts = list(ctx.gidx(m, t, m + t))
        dts = chd.EvaluationKey(ctx, uniform(g_dts)[None].contiguous(), uniform(g_dts)[None].contiguous(),
                                on_device=True, basis=(m, t, m + t))
        mm, tt = ctx.level_np(ctx.max_level)
        std = chd.EvaluationKey(ctx, uniform(kg)[None].contiguous(), uniform(kg)[None].contiguous(),
                                on_device=True, basis=(mm, tt, a))
        held += [dts, std]
        keys.set_dense_to_sparse(dts)
        keys.set_sparse_to_dense(std)
    g0 = list(ctx.gidx(*ctx.level_np(0), 0))
    ins = [ctx.import_ct(0, [uniform(g0), uniform(g0)], on_device=True, scale=ctx.scale(0)) for _ in range(B)]
    return ctx, bc, keys, held, ins


@pytest.mark.parametrize("name", BOOTS)
@pytest.mark.parametrize("min_ks", [False, True])
def test_boot_batch_equals_single_n16(cuda_ok, name, min_ks):
    ctx, bc, keys, _, ins = _setup(name)
    batch = bc.BootBatch(ins, keys, min_ks=min_ks)
    for i in range(B):
        one = bc.Boot(ins[i], keys, min_ks=min_ks).numpy()
        got = batch[i].numpy()
        assert len(one) == len(got)
        for x, y in zip(got, one):
            assert np.array_equal(x, y)
    # inputs untouched, results differ between ciphertexts
    assert not np.array_equal(batch[0].numpy()[0], batch[1].numpy()[0])
