"""Batched uneven instances: one CUDA graph per sweep for all instances, in
either schedule (one persistent launch, or the launch sequence); every
instance must end bit-identical to itself run alone."""
import numpy as np
import pytest

import bm

pytestmark = pytest.mark.gpu


def _pairs(ns, seed0=300, **kw):
    return [bm.generate(bm.gen_params(n=n, e=20 * n, seed=seed0 + i, **kw)) for i, n in enumerate(ns)]


def _alone(g, sweeps, flags=bm.BM_FLAG_NO_HUB_GEMM):
    with bm.Engine.from_pair(g, flags) as E:
        E.set_mapping(g["map0"])
        for _ in range(sweeps):
            E.sweep()
        return E.get_mapping(), E.score()


def test_batch_sweeps_match_single_instances():
    pairs = _pairs([300, 517, 800, 1203, 64])
    with bm.Batch(pairs) as B:
        B.set_mappings([g["map0"] for g in pairs])
        info = B.info()
        assert info["count"] == 5 and info["max_n"] == 1203
        c1, _ = B.sweeps(2)                      # default launch shapes
        pt, tile = B.autotune()
        assert pt in (256, 512, 1024) and tile in (32, 64)   # 1024: the one-launch sweep kernel
        c2, ms = B.sweeps(2)                     # tuned shapes, same graph replays
        maps, scores = B.get_mappings(), B.scores()
    assert (c1 > 0).all()
    for i, g in enumerate(pairs):
        m, s = _alone(g, 4)
        assert np.array_equal(maps[i], m), i
        assert scores[i] == s


def test_batch_mixed_weights_uses_one_storage_mode():
    pairs = _pairs([400, 700])
    big = dict(pairs[1])
    big["w1"] = big["w1"] * 3000   # both sides reach above 16 bits
    big["w2"] = big["w2"] * 3000
    pairs[1] = big
    with bm.Batch(pairs) as B:
        B.set_mappings([g["map0"] for g in pairs])
        B.sweeps(3)
        maps, scores = B.get_mappings(), B.scores()
    for i, g in enumerate(pairs):
        m, s = _alone(g, 3, bm.BM_FLAG_NO_HUB_GEMM | bm.BM_FLAG_FORCE_I32)
        assert np.array_equal(maps[i], m)
        assert scores[i] == s


@pytest.mark.parametrize("sched", [(True, 1024, 32), (True, 1024, 64), (False, 256, 32), (False, 512, 64)])
def test_batch_schedules_match_single_instances(sched):
    """Each schedule, set directly, gives every instance the moves it makes
    alone (the persistent launch also with 32-bit entries).  The sizes mix
    instances whose rows the persistent launch pairs on half groups with
    larger ones it does not."""
    pairs = _pairs([300, 517, 800, 1203, 64, 2600, 5200, 6100], seed0=400)
    for flags in (0, bm.BM_FLAG_FORCE_I32):
        with bm.Batch(pairs, flags) as B:
            B.set_mappings([g["map0"] for g in pairs])
            B.set_schedule(*sched)
            assert B.info()["profit_threads"] == sched[1] and B.info()["combine_tile"] == sched[2]
            c, _ = B.sweeps(3)
            maps, scores = B.get_mappings(), B.scores()
        assert (c > 0).all()
        for i, g in enumerate(pairs):
            m, s = _alone(g, 3, bm.BM_FLAG_NO_HUB_GEMM | flags)
            assert np.array_equal(maps[i], m), (sched, flags, i)
            assert scores[i] == s
