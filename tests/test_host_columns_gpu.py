"""Graphs whose column array stays in host memory (MC_HOST_COLUMNS).

The reference moves a graph that does not fit the GPU into unified memory
(include/graph_gpu.h:102-119) and runs the same kernels on it. Here the
column array goes to pinned host memory that the kernels read through the
device's mapping, chosen by the caller or by the library when the device
cannot hold the graph. Every count must equal the device-resident one and
the fixtures' golden values, bit for bit; all calls go through the C ABI.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mercury_b200 import DeviceGraph, Graph, McError, tc_count_host
from mercury_b200._ffi import MC_ERR_FORMAT
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)


def fixture(name):
    return Graph(os.path.join(GOLDEN, "graphs", name, "graph"))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_golden_counts_with_host_columns(name):
    g = fixture(name)
    with DeviceGraph(g, host_columns=True) as d:
        assert d.columns_on_host
        assert d.tc_count() == GOLD[name]["TC"]
        assert d.tc_count() == GOLD[name]["TC"]
        for k in range(1, 9):
            if f"P{k}" in GOLD[name]:
                assert d.pattern_count(k) == GOLD[name][f"P{k}"], f"P{k}"


@pytest.mark.parametrize("gen", [("rmat", 14, 16), ("rmat", 16, 16), ("cl", 40_000, 2_000)])
def test_triangles_equal_device_columns(gen):
    if gen[0] == "rmat":
        g = Graph.rmat(gen[1], gen[2], seed=3)
    else:
        g = Graph.chung_lu(gen[1], 2.1, 16.0, float(gen[2]), seed=4)
    with DeviceGraph(g) as d:
        assert not d.columns_on_host
        want = d.tc_count()
        want_shards = [d.tc_count_shard(s, 3) for s in range(3)]
    with DeviceGraph(g, host_columns=True) as h:
        assert h.tc_count() == want
        assert [h.tc_count_shard(s, 3) for s in range(3)] == want_shards
    if gen == ("rmat", 14, 16):
        assert want == orc.tc(g.rowptr, g.col)


@pytest.mark.parametrize("stage", [4096, 3 * 4096, 40_000, 1 << 20])
def test_staged_orientation_over_many_chunks(stage, monkeypatch):
    """The column array crosses to the device in chunks of whole 4096-entry
    tiles through two buffers; small chunks split rows between chunks and
    reuse each buffer many times. The DAG must equal the device-column one."""
    monkeypatch.setenv("MERCURY_STAGE_EDGES", str(stage))
    g = Graph.rmat(14, 16, seed=8)
    with DeviceGraph(g) as d:
        want = d.tc_count()
        want_dag = d.export_dag()
    with DeviceGraph(g, host_columns=True) as h:
        assert h.tc_count() == want
        got_dag = h.export_dag()
        assert np.array_equal(got_dag[0], want_dag[0]) and np.array_equal(got_dag[1], want_dag[1])
        assert h.tc_count() == want


@pytest.mark.parametrize("route", ["edge", "centers"])
def test_patterns_equal_device_columns_on_both_routes(route, monkeypatch):
    monkeypatch.setenv("MERCURY_PATTERN_KERNEL", route)
    g = Graph.rmat(9, 8, seed=11)
    with DeviceGraph(g) as d:
        want = [d.pattern_count(k) for k in range(1, 9)]
    with DeviceGraph(g, host_columns=True) as h:
        assert [h.pattern_count(k) for k in range(1, 9)] == want


def test_export_and_device_source_with_host_columns():
    import torch
    g = Graph.rmat(12, 8, seed=5)
    rp, col = np.asarray(g.rowptr), np.asarray(g.col)
    with DeviceGraph(g, host_columns=True) as h:
        r2, c2 = h.export_csr()
        assert np.array_equal(r2, rp) and np.array_equal(c2, col)
        want = h.tc_count()
    trp, tcol = torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    with DeviceGraph.from_device(trp.data_ptr(), tcol.data_ptr(), g.n, g.nnz,
                                 host_columns=True) as h2:
        assert h2.columns_on_host
        assert h2.tc_count() == want == orc.tc(rp, col)


def test_small_device_budget_chooses_host_columns(monkeypatch):
    """MERCURY_DEVICE_BYTES stands in for the device's free memory: a budget
    below the graph's in-core footprint moves the columns to the host."""
    g = Graph.rmat(13, 16, seed=2)
    want = orc.tc(g.rowptr, g.col)
    with DeviceGraph(g) as d:
        want_p4 = d.pattern_count(4)
    monkeypatch.setenv("MERCURY_DEVICE_BYTES", str(1 << 20))
    with DeviceGraph(g) as h:
        assert h.columns_on_host
        assert h.tc_count() == want
        assert h.pattern_count(4) == want_p4
    assert tc_count_host(g.rowptr, g.col) == want  # the one-shot path falls back too
    small = Graph.rmat(10, 8, seed=3)
    assert tc_count_host(small.rowptr, small.col) == orc.tc(small.rowptr, small.col)
    assert tc_count_host(g.rowptr, g.col) == want  # its cached host-column context again
    monkeypatch.setenv("MERCURY_DEVICE_BYTES", str(1 << 40))
    with DeviceGraph(g) as d:
        assert not d.columns_on_host
        assert d.tc_count() == want
    assert tc_count_host(g.rowptr, g.col) == want


@pytest.mark.parametrize("placement", ["columns", "dag"])
def test_forced_placement_counts_equal_device_placement(monkeypatch, placement):
    """MERCURY_PLACEMENT=columns / dag forces the host placements that the
    library otherwise chooses only when the graph does not fit; both give the
    in-core counts."""
    g = Graph.rmat(13, 16, seed=7)
    want = orc.tc(g.rowptr, g.col)
    with DeviceGraph(g) as d:
        want_p5 = d.pattern_count(5)
    monkeypatch.setenv("MERCURY_PLACEMENT", placement)
    with DeviceGraph(g) as h:
        assert h.columns_on_host
        assert h.dag_on_host == (placement == "dag")
        assert h.tc_count() == want
        assert h.pattern_count(5) == want_p5


def test_empty_and_edgeless_graphs_with_host_columns():
    with DeviceGraph(np.zeros(1, np.int64), np.zeros(0, np.int32), host_columns=True) as h:
        assert h.tc_count() == 0
    with DeviceGraph(np.zeros(6, np.int64), np.zeros(0, np.int32), host_columns=True) as h:
        assert h.tc_count() == 0 and h.pattern_count(3) == 0


def test_asymmetric_rows_are_refused_before_the_dag_is_written():
    """With host columns the DAG holds exactly nnz / 2 entries. A directed
    path (each row lists only its successor) keeps every entry, more than
    nnz / 2: the count is refused instead of writing past the DAG."""
    for n, stage in ((1000, 0), (50_000, 4096)):  # one chunk; 13 chunks
        if stage:
            os.environ["MERCURY_STAGE_EDGES"] = str(stage)
        try:
            rowptr = np.concatenate([np.arange(n, dtype=np.int64), [n - 1]]).astype(np.int64)
            col = np.arange(1, n, dtype=np.int32)
            with DeviceGraph(rowptr, col, host_columns=True) as h:
                with pytest.raises(McError) as ex:
                    h.tc_count()
                assert ex.value.status == MC_ERR_FORMAT
        finally:
            os.environ.pop("MERCURY_STAGE_EDGES", None)


@pytest.mark.parametrize("name", sorted(GOLD))
def test_golden_counts_with_the_dag_on_the_host(name):
    """MC_HOST_DAG: the columns and the DAG (entries and ranks) in pinned host
    memory, the counting kernels reading partner lists through the mapping."""
    g = fixture(name)
    with DeviceGraph(g, host_dag=True) as d:
        assert d.columns_on_host and d.dag_on_host
        assert d.tc_count() == GOLD[name]["TC"]
        assert d.tc_count() == GOLD[name]["TC"]


@pytest.mark.parametrize("make", [lambda: Graph.rmat(14, 16, seed=61),
                                  lambda: Graph.chung_lu(50000, 2.1, 16.0, 5000.0, seed=62)])
def test_host_dag_equals_device_dag(make):
    g = make()
    with DeviceGraph(g) as d:
        want = d.tc_count()
        drp, dcol = d.export_dag()
        parts = [d.tc_count_shard(s, 3) for s in range(3)]
    with DeviceGraph(g, host_dag=True) as h:
        assert h.tc_count() == want == orc.tc(g.rowptr, g.col)
        hrp, hcol = h.export_dag()
        assert np.array_equal(drp, hrp) and np.array_equal(dcol, hcol)
        assert [h.tc_count_shard(s, 3) for s in range(3)] == parts


def test_placement_moves_the_dag_to_the_host_when_the_device_is_too_small(monkeypatch):
    """With a device figure below the host-column footprint the library puts
    the DAG on the host too, by itself (one-shot call and handle)."""
    g = Graph.rmat(13, 16, seed=63)
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_DEVICE_BYTES", "1")
    with DeviceGraph(g) as d:
        assert d.columns_on_host and d.dag_on_host
        assert d.tc_count() == want
    assert tc_count_host(np.asarray(g.rowptr), np.asarray(g.col)) == want
