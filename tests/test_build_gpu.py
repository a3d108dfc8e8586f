"""Device CSR build from edge lists (mc_csr_build / mc_dgraph_from_edges).

The built CSR must equal the oracle's exactly (rowptr and col arrays). That
oracle is pinned to networkx on the reference's tsv2mtx.py output in
tests/test_edges.py. All calls go through the C ABI into the sm_100a kernels.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from mercury_b200 import DeviceGraph, EdgeList, Graph, McError, csr_build, dgraph_from_edges
from mercury_b200._ffi import MC_ERR_FORMAT, Timing
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

EDGES = os.path.join(GOLDEN, "edges")
META = json.load(open(os.path.join(EDGES, "edges.json")))
GOLD = json.load(open(os.path.join(GOLDEN, "golden.json")))


def assert_same_csr(g, want):
    assert np.array_equal(np.asarray(g.rowptr), want[0])
    assert np.array_equal(np.asarray(g.col), want[1])


@pytest.mark.parametrize("name", sorted(META))
@pytest.mark.parametrize("fmt", ["mtx", "tsv"])
def test_golden_edge_lists(name, fmt):
    e = EdgeList.load(os.path.join(EDGES, f"{name}.{fmt}"), fmt)
    g = e.to_graph()
    assert_same_csr(g, orc.csr_from_edges(e.src, e.dst, e.n))
    assert g.nnz == META[name]["nnz"] and g.max_degree == META[name]["max_degree"]
    g.validate(symmetry=True)


@pytest.mark.parametrize("n,m,seed", [
    (1, 0, 0), (1, 5, 1), (2, 1, 2), (3, 40, 3), (37, 500, 4), (1000, 3, 5),
    (1000, 100_000, 6), (65_539, 300_000, 7), (1 << 20, 1_000_000, 8),
])
def test_random_pairs_with_duplicates_and_self_loops(n, m, seed):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m).astype(np.int32)
    d = rng.integers(0, n, m).astype(np.int32)
    if m:
        rep = rng.integers(0, m, m // 4)
        s = np.concatenate([s, d[rep], s[rep[: m // 8]]]).astype(np.int32)   # reversed and repeated
        d = np.concatenate([d, s[rep], d[rep[: m // 8]]]).astype(np.int32)
        loops = rng.integers(0, n, m // 10 + 1).astype(np.int32)
        s = np.concatenate([s, loops]).astype(np.int32)
        d = np.concatenate([d, loops]).astype(np.int32)
    assert_same_csr(csr_build(s, d, n), orc.csr_from_edges(s, d, n))


def test_hub_rows_span_many_tiles():
    """Rows of 300k entries cross many 4096-key tiles and 512-key warp spans."""
    rng = np.random.default_rng(9)
    n = 400_000
    hub_nb = rng.permutation(n)[:300_000]
    s = np.concatenate([np.full(300_000, 17), np.full(250_000, 123_456), rng.integers(0, n, 500_000)])
    d = np.concatenate([hub_nb, rng.integers(0, n, 250_000), rng.integers(0, n, 500_000)])
    g = csr_build(s, d, n)
    assert_same_csr(g, orc.csr_from_edges(s, d, n))


def test_only_self_loops_and_isolated_tail():
    s = np.array([0, 1, 2, 2], dtype=np.int32)
    g = csr_build(s, s, 10)
    assert g.nnz == 0 and np.array_equal(g.rowptr, np.zeros(11, dtype=np.int64))
    g = csr_build(np.array([0], np.int32), np.array([1], np.int32), 10)  # 8 empty rows after
    assert g.rowptr.tolist() == [0, 1, 2] + [2] * 8 and g.col.tolist() == [1, 0]


def test_empty_inputs():
    g = csr_build(np.zeros(0, np.int32), np.zeros(0, np.int32), 0)
    assert g.n == 0 and g.nnz == 0
    g = csr_build(np.zeros(0, np.int32), np.zeros(0, np.int32), 5)
    assert g.n == 5 and g.nnz == 0 and g.rowptr.tolist() == [0] * 6


@pytest.mark.parametrize("bad", [(-1, 0), (0, 7), (7, 7), (3, -5)])
def test_ids_outside_range_are_refused(bad):
    s = np.array([0, 1, bad[0]], dtype=np.int32)
    d = np.array([1, 2, bad[1]], dtype=np.int32)
    with pytest.raises(McError) as ex:
        csr_build(s, d, 7)
    assert ex.value.status == MC_ERR_FORMAT
    with pytest.raises(McError) as ex:
        dgraph_from_edges(s, d, 7)
    assert ex.value.status == MC_ERR_FORMAT


def test_wide_ids_use_every_radix_pass():
    """n = 2^28: 57-bit keys, so the sort runs 8 passes (shift 0..56)."""
    rng = np.random.default_rng(12)
    n = 1 << 28
    s = rng.integers(0, n, 200_000).astype(np.int32)
    d = rng.integers(0, n, 200_000).astype(np.int32)
    s[:10] = n - 1
    d[10:20] = n - 1
    with dgraph_from_edges(s, d, n) as dg:
        rp, col = dg.export_csr()
    want = orc.csr_from_edges(s, d, n)
    assert np.array_equal(rp, want[0]) and np.array_equal(col, want[1])


def test_device_input_equals_host_input():
    import torch
    rng = np.random.default_rng(13)
    n, m = 5000, 60_000
    s = rng.integers(0, n, m).astype(np.int32)
    d = rng.integers(0, n, m).astype(np.int32)
    ts, td = torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda()
    torch.cuda.synchronize()
    g = csr_build(ts.data_ptr(), td.data_ptr(), n, num_edges=m, device_input=True)
    assert_same_csr(g, orc.csr_from_edges(s, d, n))
    with dgraph_from_edges(ts.data_ptr(), td.data_ptr(), n, num_edges=m, device_input=True) as dg:
        rp, col = dg.export_csr()
    assert np.array_equal(rp, np.asarray(g.rowptr)) and np.array_equal(col, np.asarray(g.col))


@pytest.mark.parametrize("scale", [12, 16])
def test_rmat_draws_build_the_generated_graph(scale):
    """Device build of the raw RMAT draws == the host generator's CSR, and
    the device graph built in place counts the same triangles."""
    e = EdgeList.rmat(scale, 16, seed=1)
    g = Graph.rmat(scale, 16, seed=1)
    t = Timing()
    assert_same_csr(csr_build(e.src, e.dst, e.n, timing=t), (np.asarray(g.rowptr), np.asarray(g.col)))
    assert t.count_ms > 0 and t.launches > 0
    with e.to_device() as dg:
        assert dg.nnz == g.nnz and dg.max_degree == g.max_degree
        assert dg.tc_count() == orc.tc(g.rowptr, g.col)


def test_fixture_round_trip_counts():
    """CSR -> edge list -> device CSR: same triangles and P3 as the fixture."""
    for name in ("rmat10", "cl3000"):
        g = Graph(os.path.join(GOLDEN, "graphs", name, "graph"))
        rp, col = np.asarray(g.rowptr), np.asarray(g.col)
        src = np.repeat(np.arange(g.n, dtype=np.int32), np.diff(rp))
        keep = src < col  # each undirected edge once
        with dgraph_from_edges(src[keep], col[keep], g.n, validate_symmetry=True) as dg:
            assert dg.tc_count() == GOLD[name]["TC"]
            if "P3" in GOLD[name]:
                assert dg.pattern_count("P3") == GOLD[name]["P3"]


@pytest.mark.parametrize("prog,base", [("converter", 1), ("converter_vidfrom0", 0)])
def test_converter_cli_writes_the_reference_triple(tmp_path, prog, base):
    exe = os.path.join(ROOT, "mercury_b200", "bin", prog)
    src = os.path.join(EDGES, "hub.mtx")
    if base == 0:  # the same graph with 0-based ids
        lines = open(src).read().splitlines()
        body = [f"{int(a) - 1} {int(b) - 1}" for a, b in (ln.split()[:2] for ln in lines[3:])]
        src = str(tmp_path / "hub0.mtx")
        open(src, "w").write("\n".join(lines[:3] + body) + "\n")
    os.makedirs(tmp_path / "g")  # converter.sh makes the output folder first
    out = subprocess.run([exe, "mtx", src, str(tmp_path / "g" / "graph"), "1", "0", "0", "0"],
                         capture_output=True, text=True, check=True).stdout
    assert "|V|: 1500" in out
    g = Graph(str(tmp_path / "g" / "graph"))
    e = EdgeList.load(os.path.join(EDGES, "hub.mtx"), "mtx")
    assert_same_csr(g, orc.csr_from_edges(e.src, e.dst, e.n))
    tc = subprocess.run([os.path.join(ROOT, "mercury_b200", "bin", "tc_challenge"),
                         str(tmp_path / "g" / "graph")], capture_output=True, text=True,
                        check=True).stdout
    assert f"total_num_triangles = {orc.tc(g.rowptr, g.col)}" in tc
