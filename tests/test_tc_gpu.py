"""Triangle count on the GPU vs the oracle and the golden fixtures.

Every count goes through the C ABI (include/mercury.h) into the sm_100a
kernels; counts are compared bit-exactly (uint64).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, csr_from_edges, relabel
from mercury_b200 import DeviceGraph, Graph, McError, tc_count_host
from mercury_b200 import _ffi
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)


def fixture(name):
    return Graph(os.path.join(GOLDEN, "graphs", name, "graph"))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_tc_matches_golden(name):
    g = fixture(name)
    with DeviceGraph(g) as d:
        assert d.tc_count() == GOLD[name]["TC"]
        assert d.tc_count() == GOLD[name]["TC"]  # second call on the same handle


@pytest.mark.parametrize("stage", ["1", "0"])
@pytest.mark.parametrize("name", ["rmat10", "cl3000", "dense400", "isolated"])
def test_device_dag_equals_oracle_orientation(name, stage, monkeypatch):
    """Pass B with each tile's entries staged in shared memory (the default)
    or written by each thread directly (MERCURY_DAG_STAGE=0)."""
    monkeypatch.setenv("MERCURY_DAG_STAGE", stage)
    g = fixture(name)
    rp, col = np.array(g.rowptr), np.array(g.col)
    with DeviceGraph(g) as d:
        d.tc_count()
        drp, dcol = d.export_dag()
        st = d.tc_stats()
    orp, ocol = orc.orient(rp, col)
    assert np.array_equal(drp, orp)
    assert np.array_equal(dcol, ocol)
    assert st["dag_edges"] == len(col) // 2
    assert st["partner_edges"] <= st["dag_edges"]


@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 1), (14, 16, 2), (16, 16, 1), (16, 32, 9)])
def test_tc_rmat_vs_oracle(scale, ef, seed):
    g = Graph.rmat(scale, ef, seed=seed)
    with DeviceGraph(g) as d:
        got = d.tc_count()
        st = d.tc_stats()
    assert got == orc.tc(g.rowptr, g.col)
    assert st["hub_tasks"] + st["leaf_tasks"] > 0


def test_dag_write_forms_give_the_same_counts(monkeypatch):
    """The hub kernel probes the DAG ranks that pass B writes: both pass-B
    forms give the oracle's count on a graph with hub tasks, in core and
    with host columns (chunked passes)."""
    g = Graph.rmat(16, 16, seed=4)
    want = orc.tc(g.rowptr, g.col)
    for stage in ("0", "1"):
        monkeypatch.setenv("MERCURY_DAG_STAGE", stage)
        with DeviceGraph(g) as d:
            assert d.tc_count() == want, stage
            assert d.tc_stats()["hub_tasks"] > 0
        with DeviceGraph(g, host_columns=True) as h:
            assert h.tc_count() == want, stage


@pytest.mark.parametrize("n,cap,seed", [(20000, 2000, 3), (200000, 50000, 1)])
def test_tc_chung_lu_vs_oracle(n, cap, seed):
    g = Graph.chung_lu(n, 2.1, 20.0, cap, seed=seed)
    with DeviceGraph(g) as d:
        assert d.tc_count() == orc.tc(g.rowptr, g.col)


def test_tc_relabel_invariance():
    g = Graph.rmat(15, 16, seed=4)
    rp, col = np.array(g.rowptr), np.array(g.col)
    perm = np.random.default_rng(1).permutation(len(rp) - 1)
    rp2, col2 = relabel(rp, col, perm)
    with DeviceGraph(rp, col) as a, DeviceGraph(rp2, col2) as b:
        assert a.tc_count() == b.tc_count()


def test_one_shot_host_entry_equals_handle_path():
    g = Graph.rmat(14, 16, seed=5)
    with DeviceGraph(g) as d:
        want = d.tc_count()
    t = _ffi.Timing()
    assert tc_count_host(g.rowptr, g.col, t) == want
    assert t.h2d_ms > 0 and t.count_ms > 0
    # a smaller graph reuses the cached buffers
    h = Graph.rmat(10, 8, seed=6)
    assert tc_count_host(h.rowptr, h.col) == orc.tc(h.rowptr, h.col)


def in_fresh_thread(body):
    """Runs body in a new thread: the one-shot call keeps a per-thread device
    context, so a new thread makes a new one (with the current settings)."""
    import threading
    errors = []

    def run():
        try:
            body()
        except BaseException as e:  # re-raised in the test's thread
            errors.append(e)

    t = threading.Thread(target=run)
    t.start()
    t.join()
    if errors:
        raise errors[0]


def test_one_shot_streams_the_columns_in_checked_chunks(monkeypatch):
    """The one-shot call copies the column array in chunks (4096 entries
    here: about 100 of them) while the contract checks and orientation
    passes run on the chunks already copied. A bad id in the last chunk or
    an unsorted row in the middle is refused, and the next call counts
    again."""
    monkeypatch.setenv("MERCURY_STAGE_EDGES", "4096")
    g = Graph.rmat(14, 16, seed=5)
    rp, col = np.asarray(g.rowptr), np.asarray(g.col)
    want = orc.tc(rp, col)
    bad_id = col.copy()
    bad_id[-1] = g.n + 5
    unsorted = col.copy()
    mid = int(np.searchsorted(rp, len(col) // 2))
    while rp[mid + 1] - rp[mid] < 2:
        mid += 1
    a = rp[mid]
    unsorted[a], unsorted[a + 1] = unsorted[a + 1], unsorted[a]

    def body():
        assert tc_count_host(rp, col) == want
        assert tc_count_host(rp, col) == want
        for bad in (bad_id, unsorted):
            with pytest.raises(McError) as ex:
                tc_count_host(rp, bad)
            assert ex.value.status == _ffi.MC_ERR_FORMAT
            assert tc_count_host(rp, col) == want

    in_fresh_thread(body)


@pytest.mark.parametrize("shards", [2, 3, 8])
def test_shard_partials_sum_to_the_count(shards):
    g = Graph.rmat(14, 16, seed=8)
    with DeviceGraph(g) as d:
        full = d.tc_count()
        parts = [d.tc_count_shard(s, shards) for s in range(shards)]
    assert sum(parts) == full
    assert all(p > 0 for p in parts)


def test_global_memory_fallback_for_large_out_lists(monkeypatch):
    """With bitmaps off and the table capped at 256 slots, owners with
    d+ > 128 take the binary-search path; the count must not change."""
    g = fixture("dense400")
    monkeypatch.setenv("MERCURY_TC_BITMAP_BITS", "0")
    monkeypatch.setenv("MERCURY_TC_TABLE_LOG2_MAX", "8")
    with DeviceGraph(g) as d:
        assert d.tc_count() == GOLD["dense400"]["TC"]
        assert d.tc_stats()["max_out_degree"] > 128


@pytest.mark.parametrize("cap", ["0", "96", "2048", "1000000"])
@pytest.mark.parametrize("make", [lambda: Graph.rmat(15, 16, seed=21),
                                  lambda: Graph.chung_lu(60000, 2.1, 20.0, 5000.0, seed=22),
                                  lambda: fixture("dense400")])
def test_hub_bitmap_and_table_paths_agree(monkeypatch, make, cap):
    """Hub owners keep N+ as a rank bitmap when rank(owner) fits the cap, as a
    cuckoo table otherwise (cap 0: tables only); every mix gives the oracle's
    count."""
    g = make()
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_BITMAP_BITS", cap)
    with DeviceGraph(g) as d:
        assert d.tc_count() == want
        assert d.tc_count() == want


@pytest.mark.parametrize("core", ["0", "1", "64", "1000", "32768", "262144"])
@pytest.mark.parametrize("make", [lambda: Graph.rmat(16, 16, seed=31),
                                  lambda: Graph.chung_lu(80000, 2.1, 24.0, 8000.0, seed=32),
                                  lambda: fixture("dense400"),
                                  lambda: fixture("k5")])
def test_dense_partners_by_core_bitmap_and(monkeypatch, make, core):
    """Long partners among the core ranks are intersected by a word-wise AND
    of the owner's bitmap with the partner's core bitmap; moving the core
    boundary (0: probes only) never changes the count."""
    g = make()
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_CORE_RANKS", core)
    with DeviceGraph(g) as d:
        assert d.tc_count() == want
        assert d.tc_count() == want
        assert sum(d.tc_count_shard(s, 3) for s in range(3)) == want


@pytest.mark.parametrize("factor", ["1", "8", "64"])
def test_dense_factor_moves_the_and_boundary(monkeypatch, factor):
    """MERCURY_TC_DENSE_FACTOR: words of a core-bitmap AND allowed per list
    entry it replaces; every boundary gives the oracle's count."""
    g = Graph.rmat(16, 16, seed=34)
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_DENSE_FACTOR", factor)
    with DeviceGraph(g) as d:
        assert d.tc_count() == want
        assert sum(d.tc_count_shard(s, 2) for s in range(2)) == want


@pytest.mark.parametrize("bits", ["0", "700", "5000"])
def test_dense_partners_with_mixed_owner_kinds(monkeypatch, bits):
    """Owners above the bitmap cap use tables and never take the AND path;
    the owners below it do; both kinds in one count give the oracle's."""
    g = Graph.rmat(15, 24, seed=33)
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_BITMAP_BITS", bits)
    monkeypatch.setenv("MERCURY_TC_CORE_RANKS", "4096")
    with DeviceGraph(g) as d:
        assert d.tc_count() == want


@pytest.mark.parametrize("cap", ["0", "1000000"])
@pytest.mark.parametrize("make", [lambda: Graph.rmat(16, 16, seed=41),
                                  lambda: Graph.chung_lu(80000, 2.1, 24.0, 8000.0, seed=42),
                                  lambda: fixture("dense400")])
def test_hub_lists_staged_by_bulk_copies(monkeypatch, make, cap):
    """MERCURY_TC_TMA=1: long partner lists reach shared memory by
    cp.async.bulk chunks (double-buffered per warp) instead of lane loads;
    bitmap owners (cap 1000000) and table owners (cap 0) both give the
    oracle's count, whole and in shards."""
    g = make()
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_TMA", "1")
    monkeypatch.setenv("MERCURY_TC_BITMAP_BITS", cap)
    with DeviceGraph(g) as d:
        assert d.tc_count() == want
        assert d.tc_count() == want
        assert sum(d.tc_count_shard(s, 3) for s in range(3)) == want


@pytest.mark.parametrize("row_stage,ranges,classes", [("1", "1", "1"), ("0", "1", "1"),
                                                      ("1", "0", "1"), ("1", "1", "0"),
                                                      ("0", "0", "0")])
@pytest.mark.parametrize("make", [lambda: Graph.rmat(16, 16, seed=51),
                                  lambda: Graph.chung_lu(80000, 2.1, 24.0, 8000.0, seed=52),
                                  lambda: fixture("dense400")])
def test_hub_row_prefetch_and_stream_forms(monkeypatch, make, row_stage, ranges, classes):
    """A hub task's row chunk reaches shared memory by a bulk copy issued one
    task ahead (MERCURY_TC_ROW_STAGE=1) or by the partner scan's own loads
    (the default); the short partner lists stream in one contiguous range per warp
    (MERCURY_TC_SHORT_RANGES=1, the default) or in interleaved windows; long
    lists of one 128-entry batch are paired before the longer ones
    (MERCURY_TC_LONG_CLASSES=1, the default) or all in row order. Each form
    gives the oracle's count on bitmap owners (cap 1000000) and table owners
    (cap 0), whole and in shards."""
    g = make()
    want = orc.tc(g.rowptr, g.col)
    monkeypatch.setenv("MERCURY_TC_ROW_STAGE", row_stage)
    monkeypatch.setenv("MERCURY_TC_SHORT_RANGES", ranges)
    monkeypatch.setenv("MERCURY_TC_LONG_CLASSES", classes)
    for cap in ("0", "1000000"):
        monkeypatch.setenv("MERCURY_TC_BITMAP_BITS", cap)
        with DeviceGraph(g) as d:
            assert d.tc_count() == want
            assert d.tc_count() == want
            assert sum(d.tc_count_shard(s, 3) for s in range(3)) == want


@pytest.mark.parametrize("row_stage", ["1", "0"])
def test_hub_row_prefetch_at_the_end_of_the_column_array(monkeypatch, row_stage):
    """The hub owner with the largest d+ renamed to the last id, so its row
    ends the column array, whose length is 2 mod 4: the prefetch copies the
    chunk up to the array's last whole 16 bytes and the partner scan loads
    the two entries after them. The count is the oracle's."""
    g = Graph.rmat(12, 16, seed=2)
    rp, col = np.array(g.rowptr), np.array(g.col)
    assert len(col) % 4 == 2
    n = len(rp) - 1
    top = int(np.argmax(np.diff(orc.orient(rp, col)[0])))
    perm = np.arange(n)
    perm[top], perm[n - 1] = n - 1, top
    rp2, col2 = relabel(rp, col, perm)
    assert np.diff(orc.orient(rp2, col2)[0])[n - 1] > 64  # a hub owner
    want = orc.tc(rp2, col2)
    monkeypatch.setenv("MERCURY_TC_ROW_STAGE", row_stage)
    with DeviceGraph(rp2, col2) as d:
        assert d.tc_count() == want
        assert sum(d.tc_count_shard(s, 2) for s in range(2)) == want


def test_empty_and_edgeless_graphs():
    with DeviceGraph(np.zeros(1, dtype=np.int64), np.zeros(0, dtype=np.int32)) as d:
        assert d.tc_count() == 0
    with DeviceGraph(np.zeros(7, dtype=np.int64), np.zeros(0, dtype=np.int32)) as d:
        assert d.tc_count() == 0
    rp, col = csr_from_edges(3, [(0, 1)])
    with DeviceGraph(rp, col) as d:
        assert d.tc_count() == 0


@pytest.mark.parametrize("rowptr,col,sym", [
    ([0, 2, 3, 4], [2, 1, 0, 0], False),    # unsorted row
    ([0, 2, 3, 4], [1, 1, 0, 0], False),    # duplicate entry
    ([0, 2, 3, 5], [1, 2, 0, 0, 2], False), # self-loop
    ([0, 1, 2], [1, 9], False),             # id out of range
    ([0, 1, 2], [1, -3], False),            # negative id
    ([0, 2, 1, 2], [1, 2], False),          # offsets not monotone
    ([0, 1, 1], [1], True),                 # asymmetric (checked on request)
])
def test_device_validation_rejects(rowptr, col, sym):
    with pytest.raises(McError) as e:
        DeviceGraph(np.array(rowptr), np.array(col), validate_symmetry=sym)
    assert e.value.status == _ffi.MC_ERR_FORMAT


def test_cli_tc_challenge_prints_reference_lines():
    import subprocess
    from conftest import ROOT
    exe = os.path.join(ROOT, "mercury_b200", "bin", "tc_challenge")
    prefix = os.path.join(GOLDEN, "graphs", "rmat10", "graph")
    out = subprocess.run([exe, prefix], capture_output=True, text=True, check=True).stdout
    assert "Triangle Counting" in out
    assert any(line.startswith("Runtime  = ") and line.endswith(" sec") for line in out.splitlines())
    assert f"total_num_triangles = {GOLD['rmat10']['TC']}" in out
