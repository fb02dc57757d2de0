"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1 set
up the process group from the launcher's environment, agree on the maximum of
their timings and meet at the barrier (the path `bench.py --gpus N` takes under
torchrun, without a GPU)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and pg is not None
    m = bench.allreduce_max(pg, 1.5 + rank)
    bench.barrier(pg)
    out.put((rank, m))
    pg.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_max():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5), (1, 2.5)]


def test_single_rank_needs_no_process_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    w, r, local, pg = bench.dist_setup()
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert bench.allreduce_max(None, 3.0) == 3.0
