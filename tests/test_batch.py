"""Batched counting: the union construction (CPU) and per-graph parity of
the captured batch launch against the single-graph path and the oracle (GPU)."""
import os

import numpy as np
import pytest

from brute import random_graph
from conftest import GOLDEN, csr_from_edges
from mercury_b200 import Batch, DeviceGraph, Graph, McError, union_csr
from mercury_b200 import _ffi
from oracle import oracle as orc


def mixed_graphs(seed, count=48):
    """Triangle jobs on RMAT/Chung-Lu graphs up to scale 12; pattern jobs on
    graphs small enough for the reference's O(sum d^3) pattern formulas."""
    rng = np.random.default_rng(seed)
    graphs, jobs = [], []
    for i in range(count):
        job = int(rng.integers(0, 9))
        if job == 0:
            kind = rng.integers(0, 3)
            if kind == 0:
                g = Graph.rmat(int(rng.integers(6, 13)), int(rng.integers(4, 17)), seed=int(rng.integers(1, 1 << 30)))
            elif kind == 1:
                g = Graph.chung_lu(int(rng.integers(500, 5000)), 2.1, 8.0, 300.0, seed=int(rng.integers(1, 1 << 30)))
            else:
                rp, col = csr_from_edges(30, random_graph(30, 0.5, int(rng.integers(1, 1000))))
                g = Graph.from_csr(rp, col)
        else:
            g = Graph.rmat(int(rng.integers(5, 8)), int(rng.integers(4, 9)), seed=int(rng.integers(1, 1 << 30)))
        graphs.append(g)
        jobs.append(job)
    return graphs, jobs


def test_union_csr_offsets():
    a = csr_from_edges(3, [(0, 1), (1, 2)])
    b = csr_from_edges(2, [(0, 1)])
    rp, col, vptr = union_csr([a, b])
    assert vptr.tolist() == [0, 3, 5]
    assert rp.tolist() == [0, 1, 3, 4, 5, 6]
    assert col.tolist() == [1, 0, 2, 1, 4, 3]
    Graph.from_csr(rp, col).validate(symmetry=True)


@pytest.mark.gpu
def test_batch_counts_equal_single_graph_counts():
    graphs, jobs = mixed_graphs(7)
    want = []
    for g, j in zip(graphs, jobs):
        with DeviceGraph(g) as d:
            want.append(d.tc_count() if j == 0 else d.pattern_count(j))
    with Batch(graphs, jobs) as b:
        got = b.count()
        assert got.tolist() == want
        assert b.count().tolist() == want  # replay of the captured launch
        choice = b.autotune()
        assert (choice[:, 0] != 0).all()
        assert b.count().tolist() == want  # tuned schedule, same counts
        assert b.last_timing.launches > 0


@pytest.mark.gpu
@pytest.mark.parametrize("leaf_max", [16, 32, 64, 128])
def test_every_autotuner_threshold_gives_single_graph_counts(monkeypatch, leaf_max):
    """Each warp/CTA threshold the autotuner can pick (owners of d+ up to
    128 on the warp kernel) gives the single-graph counts, on triangle graphs
    whose owners span d+ 1..~250."""
    graphs = [Graph.rmat(s, ef, seed=s * 7 + ef) for s, ef in ((12, 16), (14, 24), (15, 32))]
    graphs += [Graph.chung_lu(20000, 2.1, 16.0, 2000.0, seed=5)]
    jobs = [0] * len(graphs)
    want = []
    for g in graphs:
        with DeviceGraph(g) as d:
            want.append(d.tc_count())
    monkeypatch.setenv("MERCURY_BATCH_LEAF_MAX", str(leaf_max))
    with Batch(graphs, jobs) as b:
        assert b.count().tolist() == want


@pytest.mark.gpu
def test_batch_against_oracle_and_fixtures():
    names = ["k5", "star9", "petersen", "rand13", "isolated", "rmat8", "rmat10", "dense400"]
    graphs = [Graph(os.path.join(GOLDEN, "graphs", nm, "graph")) for nm in names]
    jobs = [0, 1, 4, 7, 6, 3, 0, 0]
    want = []
    for g, j in zip(graphs, jobs):
        rp, col = np.asarray(g.rowptr), np.asarray(g.col)
        want.append(orc.tc(rp, col) if j == 0 else orc.pattern(rp, col, j))
    with Batch(graphs, jobs) as b:
        assert b.count().tolist() == want


@pytest.mark.gpu
def test_batch_single_graph_and_all_patterns():
    g = Graph.rmat(7, 8, seed=11)
    graphs = [g] * 9
    jobs = list(range(9))
    rp, col = np.asarray(g.rowptr), np.asarray(g.col)
    want = [orc.tc(rp, col)] + [orc.pattern(rp, col, k) for k in range(1, 9)]
    with Batch(graphs, jobs) as b:
        assert b.count().tolist() == want


@pytest.mark.gpu
def test_batch_rejects_edges_between_graphs():
    rp = np.array([0, 1, 2], dtype=np.int64)
    col = np.array([1, 0], dtype=np.int32)
    with pytest.raises(McError) as e:
        # two graphs of one vertex each, joined by an edge
        Batch.__new__(Batch)  # (constructor below goes through the C ABI)
        import ctypes as C
        h = C.c_void_p()
        vptr = np.array([0, 1, 2], dtype=np.int64)
        jobs = np.array([0, 0], dtype=np.int32)
        _ffi.check(_ffi.lib().mc_batch_create(rp.ctypes.data, col.ctypes.data, 2, 2,
                                              vptr.ctypes.data, 2, jobs.ctypes.data, None,
                                              C.byref(h)), "batch")
    assert e.value.status == _ffi.MC_ERR_FORMAT
