"""The bounded-wait timeout paths, made to run out on purpose.

bm_test_stall(site) makes the next launch at a site take one wait that
nothing completes (CTA 0 skips an arrival, or waits for a barrier phase that
no copy or commit opens), with a short limit: no fault, trap or endless loop.
Each call must return BM_E_TIMEOUT naming the site, and the device, a fresh
context and (after a new matching) the same context must work afterwards,
with results equal to the oracle's.
"""
import numpy as np
import pytest

import bm
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("site,text", [(bm.BM_STALL_HUB_GEMM, "tensor-core hub GEMM"),
                                       (bm.BM_STALL_COMMIT, "set commit cluster barrier"),
                                       (bm.BM_STALL_COMBINE, "pair combine tile")])
def test_sweep_wait_runs_out(cfg0, site, text):
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    with bm.Engine.from_pair(g) as E:
        assert E.info()["hubs"] > 0 and g["n"] % 4 == 0   # every stalled site is on this sweep's path
        E.set_mapping(g["map0"])
        bm.test_stall(site)
        with pytest.raises(bm.BMError) as e:
            E.sweep()
        assert e.value.status == bm.BM_E_TIMEOUT
        assert text in str(e.value) and "timed out" in str(e.value)
        with pytest.raises(bm.BMError) as e:
            E.sweep()                      # the matching must be set again
        assert e.value.status == bm.BM_E_STATE
        m = g["map0"].copy()
        E.set_mapping(m)
        st = E.sweep()
        ost = O.sweep(m)
        assert st["committed"] == ost["committed"] > 0 and np.array_equal(E.get_mapping(), m)
    with bm.Engine.from_pair(g) as F:
        m = g["map0"].copy()
        F.set_mapping(m)
        F.sweep()
        O.sweep(m)
        assert np.array_equal(F.get_mapping(), m) and F.score() == O.score(m)


def test_greedy_grid_barrier_wait_runs_out():
    g = bm.generate(bm.gen_params(n=600, e=9000, seed=3))
    bm.test_stall(bm.BM_STALL_GREEDY)
    with pytest.raises(bm.BMError) as e:
        bm.greedy_match(g)
    assert e.value.status == bm.BM_E_TIMEOUT and "grid barrier wait timed out" in str(e.value)
    m, _ = bm.greedy_match(g)
    assert np.array_equal(m, oracle.greedy_match(g))


def test_mlp_gemm_wait_runs_out():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((256, bm.MLP_IN)).astype(np.float32)
    t = rng.standard_normal(256).astype(np.float32)
    with bm.Mlp(seed=4) as net:
        bm.test_stall(bm.BM_STALL_MLP_GEMM)
        with pytest.raises(bm.BMError) as e:
            net.train_step(x, t)
        assert e.value.status == bm.BM_E_TIMEOUT and "GEMM wait timed out" in str(e.value)
        loss, grads = net.train_step(x, t)     # the same object works again
    with bm.Mlp(seed=4) as ref:
        loss2, grads2 = ref.train_step(x, t)
    # float atomics in the loss and bias reductions may add in another order
    np.testing.assert_allclose(loss, loss2, rtol=1e-5)
    np.testing.assert_allclose(grads, grads2, rtol=1e-4, atol=1e-6)


def test_batch_grid_barrier_wait_runs_out():
    """The persistent batch sweep's grid barrier: the stalled sweep returns
    BM_E_TIMEOUT, the matchings must be set again, and the batch then makes
    every instance's own moves."""
    pairs = [bm.generate(bm.gen_params(n=n, e=20 * n, seed=500 + i)) for i, n in enumerate((300, 700, 1100))]
    with bm.Batch(pairs) as B:
        B.set_schedule(True, 1024, 64)
        B.set_mappings([g["map0"] for g in pairs])
        bm.test_stall(bm.BM_STALL_BATCH)
        with pytest.raises(bm.BMError) as e:
            B.sweeps(2)
        assert e.value.status == bm.BM_E_TIMEOUT and "grid barrier wait timed out" in str(e.value)
        with pytest.raises(bm.BMError) as e:
            B.sweeps(1)
        assert e.value.status == bm.BM_E_STATE
        B.set_mappings([g["map0"] for g in pairs])
        B.sweeps(2)
        maps = B.get_mappings()
    for i, g in enumerate(pairs):
        with bm.Engine.from_pair(g, bm.BM_FLAG_NO_HUB_GEMM) as E:
            E.set_mapping(g["map0"])
            E.sweep()
            E.sweep()
            assert np.array_equal(E.get_mapping(), maps[i]), i


def test_stall_hook_rejects_unknown_sites():
    with pytest.raises(bm.BMError) as e:
        bm.test_stall(99)
    assert e.value.status == bm.BM_E_INPUT
    bm.test_stall(0)
