"""bm_pair_deltas_static, the entry point that allocates nothing.

It is for callers that cannot let the library cudaMalloc (GPU memory already
handed to another allocator, or loops where an allocation's device-wide
synchronization would stall other streams).  Its deltas must equal those of
bm_pair_deltas, call after call, although every call reuses the same fixed
device array.  This file sorts last so a run that stops at the first failure
has already run every other test.
"""
import numpy as np
import pytest

import bm

pytestmark = pytest.mark.gpu


def _pairs(rng, n, k):
    a = rng.integers(1, n + 1, k).astype(np.int32)
    b = rng.integers(1, n, k).astype(np.int32)
    b = np.where(b >= a, b + 1, b).astype(np.int32)   # b != a
    return a, b


def test_static_matches_allocating_entry_point_on_two_calls_in_a_row(cfg0):
    g = cfg0
    n = g["n"]
    rng = np.random.default_rng(2024)
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(g["map0"])
        # the second call is smaller, so stale results of the first would show
        for k in (bm.BM_STATIC_MAX_PAIRS, 1234):
            a, b = _pairs(rng, n, k)
            got = E.pair_deltas_static(a, b)
            want = E.pair_deltas(a, b)
            assert np.array_equal(got, want)
        # after the matching changes, the shared array still gives fresh results
        E.sweep()
        a, b = _pairs(rng, n, 4096)
        assert np.array_equal(E.pair_deltas_static(a, b), E.pair_deltas(a, b))


def test_static_calls_allocate_nothing(cfg0):
    """Neither the context's device memory nor the device's free memory moves
    across static calls made before any allocating call; the allocating entry
    point, called afterwards, still gives the same deltas."""
    import torch
    g = cfg0
    n = g["n"]
    rng = np.random.default_rng(7)
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(g["map0"])
        a, b = _pairs(rng, n, 20_000)
        first = E.pair_deltas_static(a, b)          # looks the array's address up
        torch.cuda.synchronize()
        held = E.info()["device_bytes"]
        free0 = torch.cuda.mem_get_info()[0]
        outs = [E.pair_deltas_static(*_pairs(np.random.default_rng(s), n, bm.BM_STATIC_MAX_PAIRS))
                for s in (1, 2)]
        torch.cuda.synchronize()
        assert E.info()["device_bytes"] == held
        assert torch.cuda.mem_get_info()[0] == free0
        assert np.array_equal(first, E.pair_deltas(a, b))
        for s, o in zip((1, 2), outs):
            assert np.array_equal(o, E.pair_deltas(*_pairs(np.random.default_rng(s), n, bm.BM_STATIC_MAX_PAIRS)))


def test_static_rejects_more_pairs_than_the_fixed_array(cfg0):
    g = cfg0
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(g["map0"])
        k = bm.BM_STATIC_MAX_PAIRS + 1
        a = np.ones(k, np.int32)
        b = np.full(k, 2, np.int32)
        with pytest.raises(bm.BMError) as e:
            E.pair_deltas_static(a, b)
        assert e.value.status == bm.BM_E_INPUT
        assert "exceeds" in str(e.value)
