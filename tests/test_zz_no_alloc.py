"""chd_modup_raw_noalloc — ModUp for callers that cannot allocate device
memory (latency-critical servers, where a cudaMalloc can synchronise the
device, and hosts whose device memory belongs to another allocator or a
fixed budget).  Its scratch is a static device array of 2^21 words; the test
checks, through the C ABI, that two calls in a row give exactly the residues
of the allocating chd_modup_raw (integer work: bit-exact), at N = 2^16 and
on the small-degree path; that the call leaves the device's free memory
unchanged on a fresh context (whose arena has never grown); that a level
whose limbs exceed the static scratch, and device pointers off a 16-byte
boundary, are refused with a clear error."""
import ctypes as C
import json

import numpy as np
import pytest
import torch

import cheddar_b200 as chd
from gpu_common import param_json

pytestmark = pytest.mark.gpu


def _noalloc(ctx, level, src, dst):
    L = chd.lib()
    f = L.chd_modup_raw_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    return f(ctx.ptr, level, src.data_ptr(), dst.data_ptr())


def _uniform(ctx, level, seed):
    m, t = ctx.level_np(level)
    p = json.loads(chd.load_params("keyswitch_l24_a8.json"))
    primes = (list(reversed(p.get("terminal_primes", []))) + p["main_primes"])[:m + t]
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = torch.randint(0, 2 ** 62, (m + t, ctx.n), generator=g, device="cuda", dtype=torch.int64)
    return (r % torch.tensor(primes, device="cuda", dtype=torch.int64)[:, None]).to(torch.int32)


@pytest.mark.parametrize("log_n", [16, 13])
def test_noalloc_modup_matches_allocating_modup(cuda_ok, log_n):
    p = param_json("keyswitch_l24_a8.json", log_n)
    ctx = chd.Context(json.dumps(p))
    for call, level in enumerate((ctx.max_level, 9)):  # two calls in a row
        x = _uniform(ctx, level, 100 + call)
        beta = -(-(ctx.num_q(level)) // ctx.alpha)
        shape = (beta, ctx.num_q(level) + ctx.alpha, ctx.n)
        ref = torch.zeros(shape, dtype=torch.int32, device="cuda")
        got = torch.full(shape, -1, dtype=torch.int32, device="cuda")
        ctx.modup_raw(level, x, ref)
        ctx.synchronize()
        assert _noalloc(ctx, level, x, got) == 0, chd.lib().chd_last_error()
        ctx.synchronize()
        torch.cuda.synchronize()
        assert torch.equal(ref, got), f"level {level}"


def test_noalloc_allocates_nothing(cuda_ok):
    """On a context whose device arena is still empty the call takes no
    device memory: free memory is the same before and after it.  A warm-up
    call on another context first loads the library's kernels (lazy module
    loading allocates their code and static arrays once per process)."""
    p = json.dumps(param_json("keyswitch_l24_a8.json"))
    warm = chd.Context(p)
    lvl = warm.max_level
    beta = -(-(warm.num_q(lvl)) // warm.alpha)
    shape = (beta, warm.num_q(lvl) + warm.alpha, warm.n)
    x = _uniform(warm, lvl, 7)
    got = torch.zeros(shape, dtype=torch.int32, device="cuda")
    ref = torch.zeros(shape, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(warm, lvl, x, got) == 0, chd.lib().chd_last_error()
    warm.synchronize()
    fresh = chd.Context(p)
    fresh.synchronize()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _noalloc(fresh, lvl, x, got) == 0, chd.lib().chd_last_error()
    fresh.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes"
    fresh.modup_raw(lvl, x, ref)
    fresh.synchronize()
    assert torch.equal(ref, got)


def test_noalloc_refuses_misaligned_pointers(cuda_ok):
    ctx = chd.Context(json.dumps(param_json("keyswitch_l24_a8.json", 13)))
    lvl = ctx.max_level
    x = _uniform(ctx, lvl, 8)
    out = torch.zeros((4, ctx.num_q(lvl) + ctx.alpha, ctx.n), dtype=torch.int32, device="cuda")
    L = chd.lib()
    f = L.chd_modup_raw_noalloc
    rc = f(ctx.ptr, lvl, C.c_void_p(x.data_ptr() + 4), C.c_void_p(out.data_ptr()))
    assert rc == 1  # CHD_ERR_INVALID_ARG
    assert "16-byte aligned" in L.chd_last_error().decode()
    rc = f(ctx.ptr, lvl, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr() + 8))
    assert rc == 1


def test_noalloc_refuses_oversized_levels(cuda_ok):
    # 40 q primes at N = 2^16 need 40 * 2^16 words > 2^21: refused, no fault
    from importlib import util
    import os
    spec = util.spec_from_file_location("gen_params", os.path.join(chd.PARAM_DIR, "gen_params.py"))
    gp = util.module_from_spec(spec)
    spec.loader.exec_module(gp)
    ctx = chd.Context(json.dumps(gp.keyswitch_params(40, 8)))
    lvl = ctx.max_level
    assert ctx.num_q(lvl) == 40
    x = torch.zeros((40, ctx.n), dtype=torch.int32, device="cuda")
    out = torch.zeros((5, 48, ctx.n), dtype=torch.int32, device="cuda")
    rc = _noalloc(ctx, lvl, x, out)
    assert rc == 6  # CHD_ERR_UNSUPPORTED
    assert "exceeds the static scratch" in chd.lib().chd_last_error().decode()


def test_noalloc_refuses_digits_beyond_the_bconv_limits(cuda_ok):
    # alpha = 20 at N = 2^13 (the unfused small-degree path): a digit of 20
    # primes exceeds the base conversion's 16 sources; refused before any
    # work, like the allocating chd_modup_raw
    from importlib import util
    import os
    spec = util.spec_from_file_location("gen_params", os.path.join(chd.PARAM_DIR, "gen_params.py"))
    gp = util.module_from_spec(spec)
    spec.loader.exec_module(gp)
    ctx = chd.Context(json.dumps(gp.keyswitch_params(24, 20, log_n=13)))
    lvl = ctx.max_level
    nq = ctx.num_q(lvl)
    x = torch.zeros((nq, ctx.n), dtype=torch.int32, device="cuda")
    out = torch.zeros((-(-nq // 20), nq + 20, ctx.n), dtype=torch.int32, device="cuda")
    assert _noalloc(ctx, lvl, x, out) == 6  # CHD_ERR_UNSUPPORTED
    assert "more than 16 primes" in chd.lib().chd_last_error().decode()
    with pytest.raises(chd.CheddarError):
        ctx.modup_raw(lvl, x, out)
