"""Batched base conversion on both engines (CUDA cores: int64 multiply-adds;
tensor cores: tcgen05 INT8 4-limb GEMM with int32 accumulation) against the
oracle's kernel::ModSwitchMatrixMult restatement (src/core/ModSwitch.cu:23-171),
bit-exact.  Shapes cover the benchmark's ModUp 12 -> 4 and ModDown 4 -> 12,
the key-switching digits (8 -> 24, 9 -> 23), single-limb and 16-source
edges, and inputs at the ends of the centred range."""
import numpy as np
import pytest
import torch

import cheddar_b200 as chd
from gpu_common import pair

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


def _inputs(primes, src, npoly, n, rng, extremes=False):
    # centred residues; with extremes, half of each limb at -(q-1)/2 or (q-1)/2
    xs = []
    for _ in range(npoly):
        rows = []
        for s in src:
            h = int(primes[s]) // 2
            r = rng.integers(-h, h + 1, n)
            if extremes:
                r[: len(r) // 2] = np.where(rng.integers(0, 2, len(r) // 2) == 0, -h, h)
            rows.append(r)
        xs.append(np.stack(rows))
    return np.stack(xs).astype(np.int32)


@pytest.mark.parametrize("K,M,npoly", [(12, 4, 3), (4, 12, 3), (8, 24, 2), (9, 23, 2), (1, 1, 2), (16, 16, 2),
                                       (3, 29, 1), (13, 19, 1)])
def test_bconv_engines_bit_exact(cuda_ok, K, M, npoly):
    o, g = pair(KS)
    primes = o.all_primes()
    rng = np.random.default_rng(1000 * K + M)
    gidx = rng.permutation(len(primes))
    src, dst = gidx[:K], gidx[K:K + M]
    xt = _inputs(primes, src, npoly, o.n, rng, extremes=(K == 16))
    T = o.bconv_table(primes[src], primes[dst])
    ref = np.stack([o.bconv(xt[i], T, primes[dst]) for i in range(npoly)])
    xd = torch.from_numpy(xt).cuda()
    for engine in (chd.BCONV_CUDA_CORE, chd.BCONV_TENSOR_CORE):
        out = torch.full((npoly, M, o.n), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        g.bconv_batch(xd, src, dst, out, engine=engine, npoly=npoly)
        g.synchronize()
        assert np.array_equal(_host(out), ref), engine


def test_bconv_tensor_core_back_to_back(cuda_ok):
    # the benchmark's ModUp shape (12 -> 4) twice in a row on the stream,
    # without host synchronisation in between
    o, g = pair(KS)
    primes = o.all_primes()
    rng = np.random.default_rng(7)
    src, dst = np.arange(12), np.arange(24, 28)
    npoly = 4
    xt = _inputs(primes, src, npoly, o.n, rng)
    T = o.bconv_table(primes[src], primes[dst])
    ref = np.stack([o.bconv(xt[i], T, primes[dst]) for i in range(npoly)])
    xd = torch.from_numpy(xt).cuda()
    outs = [torch.zeros((npoly, 4, o.n), dtype=torch.int32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for out in outs:
        g.bconv_batch(xd, src, dst, out, engine=chd.BCONV_TENSOR_CORE, npoly=npoly)
    g.synchronize()
    for out in outs:
        assert np.array_equal(_host(out), ref)


def test_bconv_batch_rejects_bad_engine(cuda_ok):
    o, g = pair(KS)
    xd = torch.zeros((1, 1, o.n), dtype=torch.int32, device="cuda")
    out = torch.zeros((1, 1, o.n), dtype=torch.int32, device="cuda")
    with pytest.raises(chd.CheddarError):
        g.bconv_batch(xd, [0], [1], out, engine=7)


@pytest.mark.parametrize("npoly", [1, 8])
def test_bounded_wait_runs_out_and_context_recovers(cuda_ok, npoly):
    """The tensor-core kernel's bounded mbarrier wait gives up, without a
    fault: with the stall hook on, each CTA's first accumulator wait polls a
    barrier nothing signals (64 polls), the kernel sets the context's error
    word, drains its MMAs in flight, frees its tensor memory and returns;
    chd_context_synchronize reports CHD_ERR_CUDA with the bounded-wait
    message, clears the word, and the next launch on the same context is
    exact again.  npoly = 1 gives every CTA one iteration (the wait after the
    loop runs out), npoly = 8 several (the wait inside the loop)."""
    o, g = pair(KS)
    primes = o.all_primes()
    rng = np.random.default_rng(99)
    src, dst = np.arange(12), np.arange(24, 28)
    xt = _inputs(primes, src, npoly, o.n, rng)
    T = o.bconv_table(primes[src], primes[dst])
    ref = np.stack([o.bconv(xt[i], T, primes[dst]) for i in range(npoly)])
    xd = torch.from_numpy(xt).cuda()
    out = torch.zeros((npoly, 4, o.n), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    L = chd.lib()
    assert L.chd_debug_stall_tensor_waits(g.ptr, 64) == 0
    try:
        g.bconv_batch(xd, src, dst, out, engine=chd.BCONV_TENSOR_CORE, npoly=npoly)
        with pytest.raises(chd.CheddarError) as e:
            g.synchronize()
        assert e.value.code == 4  # CHD_ERR_CUDA
        assert "bounded wait ran out" in str(e.value)
    finally:
        assert L.chd_debug_stall_tensor_waits(g.ptr, 0) == 0
    g.synchronize()  # the error word was cleared
    out.zero_()
    torch.cuda.synchronize()
    g.bconv_batch(xd, src, dst, out, engine=chd.BCONV_TENSOR_CORE, npoly=npoly)
    g.synchronize()
    assert np.array_equal(_host(out), ref)
    assert L.chd_debug_stall_tensor_waits(g.ptr, -1) == 1  # CHD_ERR_INVALID_ARG
