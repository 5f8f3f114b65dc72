"""Two-stream key switching: a fused key switch of two or more ciphertexts
runs its halves on the context stream and on a second stream of the context.
Residues equal the one-stream pipeline's and the oracle's, for even and odd
batches, mixed levels, results written over operands and a graph capture of
the forked pipeline."""
import numpy as np
import pytest

import cheddar_b200 as chd
from gpu_common import mult_key, pair, uniform_parts

pytestmark = pytest.mark.gpu
KS = "keyswitch_l24_a8.json"


def _parts(ct):
    return [np.array(x) for x in ct.numpy()]


def _run(g, key, ga, gb, split, rescale=True):
    g.stream_split = split
    outs = g.HMultBatch(ga, gb, key, rescale=rescale)
    g.synchronize()
    return [_parts(r) for r in outs]


@pytest.mark.parametrize("levels", [[22] * 8, [22] * 5, [22, 9, 22, 5, 13, 9, 17], [3, 20]])
def test_split_equals_one_stream_and_oracle(cuda_ok, levels):
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    assert g.stream_split  # on by default
    pairs = [(lvl, uniform_parts(KS, lvl, 3100 + i), uniform_parts(KS, lvl, 3150 + i)) for i, lvl in enumerate(levels)]
    ga = [g.import_ct(lvl, a) for lvl, a, _ in pairs]
    gb = [g.import_ct(lvl, b) for lvl, _, b in pairs]
    for rescale in (True, False):
        on = _run(g, key, ga, gb, True, rescale)
        off = _run(g, key, ga, gb, False, rescale)
        for x, y in zip(on, off):
            assert all(np.array_equal(u, v) for u, v in zip(x, y))
    g.stream_split = True
    for (lvl, a, b), r in zip(pairs[:3], _run(g, key, ga[:3], gb[:3], True)):
        ref = o.hmult(lvl, a, b, (kb, ka), rescale=True)
        assert np.array_equal(r[0], ref[0]) and np.array_equal(r[1], ref[1])


def test_split_with_results_over_operands(cuda_ok):
    # results written over the first operands of their own pairs
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    lv = 22
    srcs = [(uniform_parts(KS, lv, 3300 + i), uniform_parts(KS, lv, 3350 + i)) for i in range(4)]
    ga = [g.import_ct(lv, a) for a, _ in srcs]
    gb = [g.import_ct(lv, b) for _, b in srcs]
    g.stream_split = True
    g.HMultBatch(ga, gb, key, rescale=True, res_list=ga)
    g.synchronize()
    for c, (a, b) in zip(ga, srcs):
        ref = o.hmult(lv, a, b, (kb, ka), rescale=True)
        p = _parts(c)
        assert np.array_equal(p[0], ref[0]) and np.array_equal(p[1], ref[1])


def test_graph_capture_of_forked_pipeline(cuda_ok):
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    levels = [22, 22, 15, 22, 9, 22]
    first = [(lvl, uniform_parts(KS, lvl, 3500 + i), uniform_parts(KS, lvl, 3550 + i)) for i, lvl in enumerate(levels)]
    ga = [g.import_ct(lvl, a) for lvl, a, _ in first]
    gb = [g.import_ct(lvl, b) for lvl, _, b in first]
    outs = [chd.Ciphertext(g) for _ in levels]
    g.stream_split = True
    g.HMultBatch(ga, gb, key, rescale=True, res_list=outs)
    g.synchronize()
    g.graph_begin()
    g.HMultBatch(ga, gb, key, rescale=True, res_list=outs)
    graph = g.graph_end()
    second = [(lvl, uniform_parts(KS, lvl, 3600 + i), uniform_parts(KS, lvl, 3650 + i)) for i, lvl in enumerate(levels)]
    for c, (lvl, a, _) in zip(ga, second):
        c.load(lvl, a)
    for c, (lvl, _, b) in zip(gb, second):
        c.load(lvl, b)
    g.synchronize()
    graph.launch()
    g.synchronize()
    for r, (lvl, a, b) in zip(outs, second):
        ref = o.hmult(lvl, a, b, (kb, ka), rescale=True)
        p = _parts(r)
        assert np.array_equal(p[0], ref[0]) and np.array_equal(p[1], ref[1])


@pytest.mark.parametrize("count", [2, 3, 6])
def test_moddown_batch_split(cuda_ok, count):
    # ModDown of 2 * count polynomials over Q u P: halves on two streams
    # (four or more polynomials) equal one stream and ModDown one by one
    o, g = pair(KS)
    lv = 22
    a = g.alpha
    cts = [g.import_ct(lv, uniform_parts(KS, lv, 3700 + 10 * i, num_aux=a), num_aux=a) for i in range(count)]
    g.stream_split = True
    on = [_parts(r) for r in g.ModDownBatch(cts)]
    g.stream_split = False
    off = [_parts(r) for r in g.ModDownBatch(cts)]
    g.stream_split = True
    one = [_parts(g.ModDown(c)) for c in cts]
    for x, y, z in zip(on, off, one):
        assert all(np.array_equal(u, v) and np.array_equal(u, w) for u, v, w in zip(x, y, z))


def test_ntt_batches_on_alternating_streams(cuda_ok):
    # 32 polynomials of 24 primes: more rows than one launch takes, so the
    # launches alternate between the two streams; residues equal one stream,
    # the oracle's transform, and the inverse returns the input
    import torch
    o, g = pair(KS)
    lvl = g.max_level
    m, t = g.level_np(lvl)
    x = np.stack([o.uniform(4000 + i, lvl) for i in range(32)])
    outs = {}
    for on in (True, False):
        g.stream_split = on
        dev = torch.from_numpy(x.view(np.int32).copy()).cuda()
        g.ntt_raw(m, t, 0, dev, mont=True, count=32)
        g.synchronize()
        outs[on] = dev.cpu().numpy().view(np.uint32).copy()
        g.intt_raw(m, t, 0, dev, mont=True, count=32)
        g.synchronize()
        assert np.array_equal(dev.cpu().numpy().view(np.uint32), x)
    g.stream_split = True
    assert np.array_equal(outs[True], outs[False])
    for i in (0, 13, 31):
        assert np.array_equal(outs[True][i], o.ntt(lvl, x[i], mont=True))


def test_failed_half_leaves_context_usable(cuda_ok):
    # a key with too few digits makes the first half of a split batch fail
    # after the fork: the call returns the error, the join is still
    # recorded, and the next batch on the same context is right
    o, g = pair(KS)
    (kb, ka), key = mult_key(KS)
    lvl = 22
    pairs = [(uniform_parts(KS, lvl, 3800 + i), uniform_parts(KS, lvl, 3850 + i)) for i in range(4)]
    ga = [g.import_ct(lvl, a) for a, _ in pairs]
    gb = [g.import_ct(lvl, b) for _, b in pairs]
    _, basis = key.info()  # the key basis, one digit only
    short = chd.EvaluationKey(g, np.ascontiguousarray(kb[:1]), np.ascontiguousarray(ka[:1]), basis=basis)
    g.stream_split = True
    with pytest.raises(chd.CheddarError) as err:
        g.HMultBatch(ga, gb, short, rescale=True)
    assert "too few digits" in str(err.value)
    g.synchronize()
    outs = g.HMultBatch(ga, gb, key, rescale=True)
    g.synchronize()
    for r, (a, b) in zip(outs, pairs):
        ref = o.hmult(lvl, a, b, (kb, ka), rescale=True)
        p = _parts(r)
        assert np.array_equal(p[0], ref[0]) and np.array_equal(p[1], ref[1])
