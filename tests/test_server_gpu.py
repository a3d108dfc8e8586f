"""Serving with continuous batching: every result equals the single-graph
result, alone and in a mix; resident cache, HBM-budget refusal, overlap."""
import threading
import time

import numpy as np
import pytest

from mercury_b200 import DeviceGraph, Graph, McError, Server
from mercury_b200 import _ffi

pytestmark = pytest.mark.gpu


def small_mix(seed, count):
    rng = np.random.default_rng(seed)
    graphs, jobs = [], []
    for _ in range(count):
        job = int(rng.integers(0, 9))
        scale = int(rng.integers(6, 12)) if job == 0 else int(rng.integers(5, 8))
        graphs.append(Graph.rmat(scale, int(rng.integers(4, 12)), seed=int(rng.integers(1, 1 << 30))))
        jobs.append(job)
    return graphs, jobs


def plain(g, job):
    with DeviceGraph(g) as d:
        return d.tc_count() if job == 0 else d.pattern_count(job)


def test_each_result_is_the_same_alone_and_in_the_mix():
    graphs, jobs = small_mix(3, 120)
    want = [plain(g, j) for g, j in zip(graphs, jobs)]
    with Server(8 << 30, max_batch=64, workers=2) as s:
        # alone: one request in flight at a time
        alone = []
        for g, j in zip(graphs[:20], jobs[:20]):
            alone.append(s.wait(s.submit(g, j))[0])
        assert alone == want[:20]
        # in the mix: everything submitted at once, from two threads
        tickets = [None] * len(graphs)

        def submit(lo, hi):
            for i in range(lo, hi):
                tickets[i] = s.submit(graphs[i], jobs[i])
        threads = [threading.Thread(target=submit, args=(0, 60)),
                   threading.Thread(target=submit, args=(60, 120))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        mixed = [s.wait(t)[0] for t in tickets]
        st = s.stats()
    assert mixed == want
    assert st["completed"] == 140 and st["failed"] == 0
    assert st["max_batch_seen"] > 1  # requests were coalesced


def test_work_cap_of_one_runs_every_request_alone(monkeypatch):
    """MERCURY_SERVE_BATCH_WORK=1: every request's estimated work is above
    the cap, so each runs in a batch of its own; the results equal the plain
    path's."""
    monkeypatch.setenv("MERCURY_SERVE_BATCH_WORK", "1")
    graphs, jobs = small_mix(5, 24)
    want = [plain(g, j) for g, j in zip(graphs, jobs)]
    with Server(8 << 30, max_batch=64, workers=2) as s:
        tickets = [s.submit(g, j) for g, j in zip(graphs, jobs)]
        got = [s.wait(t)[0] for t in tickets]
        st = s.stats()
    assert got == want
    assert st["max_batch_seen"] == 1 and st["batches"] == 24


def test_resident_cache_serves_keyed_graphs_without_arrays():
    g = Graph.rmat(10, 8, seed=5)
    want = plain(g, 0)
    with Server(4 << 30) as s:
        first = s.wait(s.submit(g, "TC", key=77))[0]
        again = s.wait(s.submit(None, "TC", key=77))[0]
        p4 = s.wait(s.submit(None, "P4", key=77))[0]
        st = s.stats()
    assert first == again == want
    assert p4 == plain(g, 4)
    assert st["cache_hits"] >= 2 and st["cached_graphs"] == 1


def test_budget_refuses_requests_that_cannot_fit():
    g = Graph.rmat(12, 16, seed=2)
    with Server(1 << 20) as s:  # 1 MiB
        t = s.submit(g, "TC")
        with pytest.raises(McError) as e:
            s.wait(t)
        assert e.value.status == _ffi.MC_ERR_BUDGET
        small = Graph.rmat(4, 2, seed=1)
        assert s.wait(s.submit(small, "TC"))[0] == plain(small, 0)


def test_arrivals_during_running_batches_overlap():
    graphs, jobs = small_mix(9, 200)
    want = [plain(g, j) for g, j in zip(graphs, jobs)]
    with Server(8 << 30, max_batch=32, workers=3) as s:
        tickets = []
        for i, (g, j) in enumerate(zip(graphs, jobs)):
            tickets.append(s.submit(g, j))
            if i % 25 == 0:
                time.sleep(0.002)  # arrivals spread over the running batches
        got = [s.wait(t) for t in tickets]
        st = s.stats()
    assert [c for c, _ in got] == want
    assert st["batches"] >= 3
    assert all(lat > 0 for _, lat in got)
