"""Multi-rank host logic on CPU: two `gloo` ranks (spawned processes, 127.0.0.1).

Checks what runs between ranks when independent work is split over GPUs: the timing reduction
(max of times, sum of counts), the deterministic partition every rank computes alone, each rank
serving its share of a request stream (simulated device), and the statistics gathered after.
"""
import os
import socket
import sys

import pytest

from epp.ranks import Ranks, partition

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_partition_balanced_deterministic():
    w = [5, 1, 9, 3, 3, 7, 2, 8, 1, 4]
    shares = partition(w, 3)
    assert sorted(i for s in shares for i in s) == list(range(len(w)))
    loads = [sum(w[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(w)
    assert shares == partition(w, 3)
    assert partition(w, 1) == [list(range(len(w)))]
    assert partition([], 2) == [[], []]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    for p in (ROOT, os.path.join(ROOT, "etherparallelparticles.jl_b200"), HERE):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    try:
        from epp import serve
        from epp.ranks import Ranks, partition
        from test_serve import FakeBackend, TickClock, fake_runs
        rk = Ranks.from_env()
        rk.init("gloo", timeout_s=60)
        ms, counts = rk.reduce_timing(10.0 + rank, [100 * (rank + 1), 1])
        sizes = [20000, 5000, 50000, 10000, 30000, 8000, 12000, 40000]
        arrivals = [0.0005 * i for i in range(len(sizes))]
        shares = partition(sizes, world)
        mine = shares[rank]
        clock = TickClock()
        runs = fake_runs([sizes[i] for i in mine], [arrivals[i] for i in mine])
        st = serve.Server(FakeBackend(clock), clock=clock, idle_wait=0.0).run(runs)
        every = rk.gather({"rank": rank, "share": mine, "completed": st["completed"]})
        rk.finish()
        q.put((rank, ms, counts, shares, every, None))
    except Exception as exc:  # reported to the parent
        q.put((rank, None, None, None, None, repr(exc)))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            r = q.get(timeout=120)
            out[r[0]] = r
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for r in (0, 1):
        rank, ms, counts, shares, every, err = out[r]
        assert err is None, err
        assert ms == 11.0                       # max over ranks
        assert counts == [300.0, 2.0]           # sums over ranks
        assert shares == out[0][3]              # both ranks computed the same split
        assert [e["rank"] for e in every] == [0, 1]
        assert sorted(i for e in every for i in e["share"]) == list(range(8))
        assert sum(e["completed"] for e in every) == 8


def test_single_rank_is_identity():
    rk = Ranks()
    assert rk.reduce_timing(3.5, [7]) == (3.5, [7.0])
    assert rk.gather({"a": 1}) == [{"a": 1}]
