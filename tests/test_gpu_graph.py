"""Mixed-level HMult batches (at N = 2^16 one pipeline over every level: a
launch per stage, the key-switch row pass taking several levels per launch)
and CUDA-graph capture of library calls: a captured batch replayed on refreshed inputs and
a captured bootstrap replayed give the oracle's residues, bit for bit."""
import numpy as np
import pytest

import cheddar_b200 as chd
from boot_oracle import Ct, run_program
from gpu_common import mult_key, pair, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"
LEVELS = [22, 9, 22, 5, 13, 9]


def _oracle_hmults(o, kb_ka, pairs):
    return [o.hmult(lvl, a, b, kb_ka, rescale=True) for lvl, a, b in pairs]


def test_mixed_level_batch(cuda_ok):
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    pairs = [(lvl, uniform_parts(KS, lvl, 900 + i), uniform_parts(KS, lvl, 950 + i)) for i, lvl in enumerate(LEVELS)]
    ga = [g.import_ct(lvl, a) for lvl, a, _ in pairs]
    gb = [g.import_ct(lvl, b) for lvl, _, b in pairs]
    outs = g.HMultBatch(ga, gb, key, rescale=True)
    for r, ref in zip(outs, _oracle_hmults(o, (kb, ka), pairs)):
        parts = r.numpy()
        assert np.array_equal(parts[0], ref[0]) and np.array_equal(parts[1], ref[1])


def test_mixed_level_batch_beyond_launch_limits(cuda_ok):
    # 18 pairs at 18 distinct levels: more ciphertexts than one row-pass
    # launch takes (16) and more levels than one launch describes (8)
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    levels = [22, 1, 3, 5, 7, 9, 11, 13, 15, 17, 19, 21, 2, 4, 6, 8, 10, 12]
    pairs = [(lvl, uniform_parts(KS, lvl, 1300 + i), uniform_parts(KS, lvl, 1350 + i)) for i, lvl in enumerate(levels)]
    ga = [g.import_ct(lvl, a) for lvl, a, _ in pairs]
    gb = [g.import_ct(lvl, b) for lvl, _, b in pairs]
    for rescale in (True, False):
        outs = g.HMultBatch(ga, gb, key, rescale=rescale)
        singles = [g.HMult(x, y, key, rescale=rescale) for x, y in zip(ga, gb)]
        for r, s1, (lvl, _, _) in zip(outs, singles, pairs):
            ri, si = r.info(), s1.info()
            assert (ri["num_main"], ri["num_ter"]) == tuple(g.level_np(lvl - 1 if rescale else lvl))
            assert ri == si
            for x, y in zip(r.numpy(), s1.numpy()):
                assert np.array_equal(x, y)
    for r, ref in zip(g.HMultBatch(ga[:6], gb[:6], key, rescale=True), _oracle_hmults(o, (kb, ka), pairs[:6])):
        parts = r.numpy()
        assert np.array_equal(parts[0], ref[0]) and np.array_equal(parts[1], ref[1])


def test_graph_replay_mixed_batch(cuda_ok):
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    first = [(lvl, uniform_parts(KS, lvl, 1100 + i), uniform_parts(KS, lvl, 1150 + i)) for i, lvl in enumerate(LEVELS)]
    ga = [g.import_ct(lvl, a) for lvl, a, _ in first]
    gb = [g.import_ct(lvl, b) for lvl, _, b in first]
    outs = [chd.Ciphertext(g) for _ in LEVELS]
    g.HMultBatch(ga, gb, key, rescale=True, res_list=outs)  # sizes results and scratch
    g.synchronize()
    g.graph_begin()
    g.HMultBatch(ga, gb, key, rescale=True, res_list=outs)
    graph = g.graph_end()
    # new inputs into the same buffers, then replay twice
    second = [(lvl, uniform_parts(KS, lvl, 1200 + i), uniform_parts(KS, lvl, 1250 + i)) for i, lvl in enumerate(LEVELS)]
    for c, (lvl, a, _) in zip(ga, second):
        c.load(lvl, a)
    for c, (lvl, _, b) in zip(gb, second):
        c.load(lvl, b)
    g.synchronize()
    graph.launch()
    graph.launch()
    g.synchronize()
    for r, ref in zip(outs, _oracle_hmults(o, (kb, ka), second)):
        parts = r.numpy()
        assert np.array_equal(parts[0], ref[0]) and np.array_equal(parts[1], ref[1])


def test_graph_replay_bootstrap(cuda_ok):
    from test_gpu_bootstrap import _setup
    o, g, bc, s, mk, ck, rks, keys = _setup()
    rng = np.random.default_rng(77)
    msg = (rng.random(o.n // 2) * 2 - 1) + 1j * (rng.random(o.n // 2) * 2 - 1)
    sc0 = o.scale(0)
    bx, ax = o.encrypt(6, s, 0, o.encode(0, sc0, msg))
    ct = g.import_ct(0, [bx, ax], sc0)
    res = chd.Ciphertext(g)
    bc.Boot(ct, keys, res=res)
    g.synchronize()
    g.graph_begin()
    bc.Boot(ct, keys, res=res)
    graph = g.graph_end()
    bx2, ax2 = o.encrypt(7, s, 0, o.encode(0, sc0, msg * 0.5))
    ct.load(0, [bx2, ax2], sc0)
    g.synchronize()
    graph.launch()
    g.synchronize()
    ref = run_program(o, bc.json(), Ct(0, [bx2, ax2], sc0), mult_key=mk, conj_key=ck, rot_keys=rks,
                      lts=bc.transforms())
    parts = res.numpy()
    assert np.array_equal(parts[0], ref.parts[0]) and np.array_equal(parts[1], ref.parts[1])
