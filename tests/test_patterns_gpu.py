"""P1..P8 on the GPU vs the golden fixtures, the reference programs' outputs
and the oracle (bit-exact uint64), through the C ABI."""
import json
import os
import sys

import numpy as np
import pytest

from brute import random_graph
from conftest import GOLDEN, csr_from_edges, relabel
from mercury_b200 import DeviceGraph, Graph
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)
with open(os.path.join(GOLDEN, "reference_counts.json")) as f:
    REF = json.load(f)["fixtures"]

PATTERN_FIXTURES = sorted(k for k in GOLD if "P1" in GOLD[k])


@pytest.mark.parametrize("name", PATTERN_FIXTURES)
@pytest.mark.parametrize("k", range(1, 9))
def test_pattern_matches_golden_and_reference(name, k):
    g = Graph(os.path.join(GOLDEN, "graphs", name, "graph"))
    with DeviceGraph(g) as d:
        got = d.pattern_count(k)
    assert got == GOLD[name][f"P{k}"]
    assert got == REF[name][f"P{k}"]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_patterns_random_dense_vs_oracle(seed):
    rp, col = csr_from_edges(40, random_graph(40, 0.3, seed))
    with DeviceGraph(rp, col) as d:
        for k in range(1, 9):
            assert d.pattern_count(k) == orc.pattern(rp, col, k), k


_DENSE = {}


def dense_case(n, p, seed):
    """Dense seeded graph and its oracle counts (computed once per module)."""
    if (n, p, seed) not in _DENSE:
        rp, col = csr_from_edges(n, random_graph(n, p, seed))
        _DENSE[(n, p, seed)] = (rp, col, [orc.pattern(rp, col, k) for k in range(1, 9)])
    return _DENSE[(n, p, seed)]


@pytest.mark.parametrize("n,p,seed", [(120, 0.5, 11), (200, 0.6, 12)])
@pytest.mark.parametrize("sets", ["1", "0"])
def test_patterns_dense_hash_and_search_forms_vs_oracle(monkeypatch, n, p, seed, sets):
    """Dense graphs: common neighbourhoods above 32 (the P8 bitmask limit)
    and degrees up to 138. The shared-memory set forms (sets=1) and the
    binary-search forms (MERCURY_PATTERN_SETS=0) both give the oracle's
    counts."""
    monkeypatch.setenv("MERCURY_PATTERN_SETS", sets)
    monkeypatch.setenv("MERCURY_PATTERN_KERNEL", "edge")
    rp, col, want = dense_case(n, p, seed)
    with DeviceGraph(rp, col) as d:
        assert [d.pattern_count(k) for k in range(1, 9)] == want


@pytest.mark.parametrize("make", [lambda: Graph.chung_lu(30000, 2.1, 12.0, 900.0, seed=7),
                                  lambda: Graph.rmat(13, 16, seed=5)])
def test_hash_set_forms_equal_search_forms(monkeypatch, make):
    """Hubs of degree up to 900 put some edges past the 512-key table; both
    forms agree on every pattern of the warp-per-edge route."""
    g = make()
    monkeypatch.setenv("MERCURY_PATTERN_KERNEL", "edge")
    with DeviceGraph(g) as d:
        fast = [d.pattern_count(k) for k in range(1, 9)]
        monkeypatch.setenv("MERCURY_PATTERN_SETS", "0")
        slow = [d.pattern_count(k) for k in range(1, 9)]
    assert fast == slow


def test_patterns_chung_lu_vs_oracle():
    g = Graph.chung_lu(4000, 2.1, 10.0, 200.0, seed=9)
    rp, col = np.array(g.rowptr), np.array(g.col)
    with DeviceGraph(g) as d:
        for k in (1, 4, 6, 8):
            assert d.pattern_count(k) == orc.pattern(rp, col, k), k


def center_class_graph():
    """One center per degree class of the bitmap kernels (20, 50, 100, 200,
    450, 900) and a hub of degree 1100 (above the bitmap limit), attached to a
    pool of 3,993 vertices, with 2d chords inside each center's neighbourhood
    and 8,000 random pool edges (seeded numpy)."""
    rng = np.random.default_rng(2024)
    n = 4000
    centers = [(0, 20), (1, 50), (2, 100), (3, 200), (4, 450), (5, 900), (6, 1100)]
    pool = np.arange(7, n)
    edges = []
    for c, d in centers:
        nb = rng.choice(pool, d, replace=False)
        edges += [(c, int(x)) for x in nb]
        # chords inside the neighbourhood: triangles and 4-cliques through c
        i, j = rng.integers(0, d, 2 * d), rng.integers(0, d, 2 * d)
        edges += [(int(nb[x]), int(nb[y])) for x, y in zip(i, j)]
    a, b = rng.integers(7, n, 8000), rng.integers(7, n, 8000)
    edges += [(int(x), int(y)) for x, y in zip(a, b)]
    return csr_from_edges(n, edges)


@pytest.mark.parametrize("route", ["default", "centers", "edge"])
def test_center_classes_and_big_centers_vs_oracle(monkeypatch, route):
    """On the center route, centers of degree <= 1024 go through the bitmap
    kernels (every class here) and larger ones through the warp-per-edge
    kernel; MERCURY_PATTERN_KERNEL forces one route for every pattern. All
    routes give the oracle's counts (tests/golden/make_center_golden.py)."""
    with open(os.path.join(GOLDEN, "center_counts.json")) as f:
        want = json.load(f)
    if route != "default":
        monkeypatch.setenv("MERCURY_PATTERN_KERNEL", route)
    rp, col = center_class_graph()
    assert len(col) == want["nnz"]
    with DeviceGraph(rp, col) as d:
        for k in range(1, 9):
            assert d.pattern_count(k) == want[f"P{k}"], k


@pytest.mark.parametrize("seed", [4])
def test_center_patterns_chung_lu_vs_oracle(seed):
    g = Graph.chung_lu(6000, 2.1, 8.0, 300.0, seed=seed)
    rp, col = np.array(g.rowptr), np.array(g.col)
    with DeviceGraph(g) as d:
        for k in (1, 3, 7):
            assert d.pattern_count(k) == orc.pattern(rp, col, k), k


@pytest.mark.parametrize("make", [lambda: Graph.chung_lu(30000, 2.1, 12.0, 900.0, seed=7),
                                  lambda: Graph.rmat(13, 16, seed=5)])
def test_center_route_equals_edge_route(monkeypatch, make):
    """Every pattern: the bitmap route equals the warp-per-edge route, on
    graphs with centers in every class (too large for the oracle here)."""
    g = make()
    with DeviceGraph(g) as d:
        monkeypatch.setenv("MERCURY_PATTERN_KERNEL", "centers")
        fast = [d.pattern_count(k) for k in range(1, 9)]
        monkeypatch.setenv("MERCURY_PATTERN_KERNEL", "edge")
        slow = [d.pattern_count(k) for k in range(1, 9)]
    assert fast == slow


def test_pattern_relabel_invariance():
    g = Graph.rmat(9, 8, seed=3)
    rp, col = np.array(g.rowptr), np.array(g.col)
    rp2, col2 = relabel(rp, col, np.random.default_rng(4).permutation(len(rp) - 1))
    with DeviceGraph(rp, col) as a, DeviceGraph(rp2, col2) as b:
        for k in range(1, 9):
            assert a.pattern_count(k) == b.pattern_count(k), k


def test_pattern_repeat_and_bad_id():
    g = Graph(os.path.join(GOLDEN, "graphs", "rmat8", "graph"))
    with DeviceGraph(g) as d:
        first = [d.pattern_count(k) for k in range(1, 9)]
        again = [d.pattern_count(k) for k in range(1, 9)]
        assert first == again
        with pytest.raises(Exception):
            d.pattern_count(9)


def test_cli_sm_prints_reference_lines():
    import subprocess
    from conftest import ROOT
    exe = os.path.join(ROOT, "mercury_b200", "bin", "sm")
    prefix = os.path.join(GOLDEN, "graphs", "rmat8", "graph")
    out = subprocess.run([exe, prefix, "P4"], capture_output=True, text=True, check=True).stdout
    assert "Total runtime  = " in out
    assert f"total_num_triangles = {GOLD['rmat8']['P4']}" in out


@pytest.mark.parametrize("route", ["default", "centers", "edge"])
@pytest.mark.parametrize("shards", [2, 3])
def test_pattern_shards_sum_to_the_count(monkeypatch, route, shards):
    """mc_pattern_count_shard: the partial counts of all shards (centers by
    id, remaining edge and star tasks round-robin) sum to the count mod 2^64,
    on every route, including the large centers of the warp-per-edge kernel."""
    if route != "default":
        monkeypatch.setenv("MERCURY_PATTERN_KERNEL", route)
    rp, col = center_class_graph()
    with DeviceGraph(rp, col) as d:
        for k in range(1, 9):
            full = d.pattern_count(k)
            parts = [d.pattern_count_shard(k, s, shards) for s in range(shards)]
            assert sum(parts) % (1 << 64) == full, k
        with pytest.raises(Exception):
            d.pattern_count_shard(1, shards, shards)


@pytest.mark.parametrize("route", ["edge", "centers"])
def test_sliced_launches_equal_one_launch(monkeypatch, route):
    """Counting in slices of the task range (each slice a launch with its own
    queue) gives the same counts as one launch per kernel, on both routes."""
    g = Graph.chung_lu(30000, 2.1, 12.0, 2000.0, seed=9)
    monkeypatch.setenv("MERCURY_PATTERN_KERNEL", route)
    with DeviceGraph(g) as d:
        monkeypatch.setenv("MERCURY_PATTERN_SLICE", "0")
        whole = [d.pattern_count(k) for k in range(1, 9)]
        monkeypatch.setenv("MERCURY_PATTERN_SLICE", "1")
        monkeypatch.setenv("MERCURY_PATTERN_SLICE_MS", "0.2")  # many small slices
        sliced = [d.pattern_count(k) for k in range(1, 9)]
        assert d.last_timing.launches > 8
    assert sliced == whole


def test_budget_stops_between_slices_and_counts_within_it():
    g = Graph.chung_lu(30000, 2.1, 12.0, 2000.0, seed=9)
    with DeviceGraph(g) as d:
        want = d.pattern_count(5)
        got, frac = d.pattern_count_budget(5, 60000.0)
        assert got == want and frac == 1.0
        # A budget below one slice: the first slice runs (one task per
        # resident warp), then the count stops with the rest undone.
        got, frac = d.pattern_count_budget(5, 1e-6)
        assert got is None and 0.0 < frac < 1.0
        assert d.pattern_count(5) == want  # the handle stays usable


def test_pattern_bench_graph_counts_equal_committed_oracle():
    """The graph bench.py --mode patterns counts (Chung-Lu n 100,000, mean 10,
    cap 200, seed 1): all eight counts equal the oracle's, committed by
    tests/golden/make_pattern_golden.py."""
    with open(os.path.join(GOLDEN, "pattern_counts.json")) as f:
        rec = json.load(f)["chung_lu_n100000_mean10_cap200_seed1"]
    g = Graph.chung_lu(100000, 2.1, 10.0, 200.0, seed=1)
    assert g.nnz // 2 == rec["m"]
    with DeviceGraph(g) as d:
        for k in range(1, 9):
            assert d.pattern_count(k) == rec["counts"][f"P{k}"], k


@pytest.mark.parametrize("route", ["default", "centers", "edge"])
def test_power_law_graph_with_hubs_counts_equal_committed_oracle(monkeypatch, route):
    """The shape of the pattern benchmark graph (Chung-Lu gamma 2.1, mean 20,
    weight cap 50,000) at 5,000 vertices, small enough for the literal oracle:
    hubs of degree 2,187, 1,525 and 1,173 (above the 1,024 limit of the
    bitmap kernels, P1's hub tasks included). All eight counts equal the
    oracle's, committed by tests/golden/make_pattern_golden.py, on every
    route and in sliced launches."""
    with open(os.path.join(GOLDEN, "pattern_counts.json")) as f:
        rec = json.load(f)["chung_lu_n5000_mean20_cap50000_seed1"]
    g = Graph.chung_lu(5000, 2.1, 20.0, 50000.0, seed=1)
    assert g.nnz // 2 == rec["m"]
    deg = np.diff(np.asarray(g.rowptr))
    assert int(deg.max()) == rec["max_degree"] and int((deg > 1024).sum()) == 3
    if route != "default":
        monkeypatch.setenv("MERCURY_PATTERN_KERNEL", route)
    with DeviceGraph(g) as d:
        for k in range(1, 9):
            assert d.pattern_count(k) == rec["counts"][f"P{k}"], k
        monkeypatch.setenv("MERCURY_PATTERN_SLICE", "1")
        monkeypatch.setenv("MERCURY_PATTERN_SLICE_MS", "0.2")  # many small slices
        for k in (1, 2, 5, 8):
            assert d.pattern_count(k) == rec["counts"][f"P{k}"], ("sliced", k)


@pytest.mark.parametrize("words", [None, "2048"])
@pytest.mark.parametrize("make", [lambda: Graph.chung_lu(30000, 2.1, 12.0, 900.0, seed=7),
                                  lambda: Graph.rmat(10, 16, seed=5)])
def test_center_route_two_hop_rows_equal_per_edge_rows(monkeypatch, make, words):
    """The center route's outer rows R(y) = N(y) & N0 come from the center's
    two-hop rows (built once per center) or are built per edge
    (MERCURY_HOP_ROWS=0); with a small scratch share (words = 2048) the
    larger centers fall back to per-edge rows within the same launch.  Every
    outer pattern gives the same counts either way, and the oracle's."""
    g = make()
    monkeypatch.setenv("MERCURY_PATTERN_KERNEL", "centers")
    if words:
        monkeypatch.setenv("MERCURY_HOP_WORDS", words)
    outer = (2, 4, 5, 6, 8)
    with DeviceGraph(g) as d:
        hop = [d.pattern_count(k) for k in outer]
        monkeypatch.setenv("MERCURY_HOP_ROWS", "0")
        per_edge = [d.pattern_count(k) for k in outer]
    assert hop == per_edge
    if g.n <= 5000:
        assert hop == [orc.pattern(g.rowptr, g.col, k) for k in outer]


@pytest.mark.parametrize("hub,lane_scan", [("1", "64"), ("1", "0"), ("1", "100000"), ("0", "64")])
def test_p1_large_centers_by_bitmap_tasks(monkeypatch, hub, lane_scan):
    """P1 on centers above degree 1,024: one CTA per (center, 256 edges)
    with the center's neighbourhood as an id bitmap (MERCURY_HUB_P1=1, the
    default) or the warp-per-edge kernel (=0); both give the oracle's counts,
    whole and in shards, on a graph with a vertex of degree 20,000 and on a
    Chung-Lu graph with hubs up to ~5,000."""
    sys.path.insert(0, GOLDEN)
    from make_hub_golden import hub_graph
    with open(os.path.join(GOLDEN, "hub_counts.json")) as f:
        hub_want = json.load(f)["counts"]["P1"]
    monkeypatch.setenv("MERCURY_HUB_P1", hub)
    monkeypatch.setenv("MERCURY_HUB_LANE_SCAN", lane_scan)
    rp, col = hub_graph()
    with DeviceGraph(rp, col) as d:
        assert d.pattern_count(1) == hub_want
    g = Graph.chung_lu(60000, 2.1, 16.0, 5000.0, seed=23)
    want = orc.pattern_fast(g.rowptr, g.col, 1)
    with DeviceGraph(g) as d:
        assert d.pattern_count(1) == want
        assert sum(d.pattern_count_shard(1, s, 3) for s in range(3)) % (1 << 64) == want


CLIQUE_FIXTURES = sorted(k for k in GOLD if "P7" in GOLD[k] and "P8" in GOLD[k])


def test_clique_route_on_fixtures_and_random_graphs(monkeypatch):
    """MERCURY_CLIQUE_ROUTE=cliques: P7 and P8 from triangle, K4 and K5 counts
    listed on the degree-ordered DAG (inclusion-exclusion of the formulas'
    per-edge sets) equal the golden counts, the oracle on random graphs of
    rising density, and the sum of their shards (mod 2^64)."""
    monkeypatch.setenv("MERCURY_CLIQUE_ROUTE", "cliques")
    for name in CLIQUE_FIXTURES:
        g = Graph(os.path.join(GOLDEN, "graphs", name, "graph"))
        with DeviceGraph(g) as d:
            for k in (7, 8):
                assert d.pattern_count(k) == GOLD[name][f"P{k}"], (name, k)
                parts = [d.pattern_count_shard(k, s, 3) for s in range(3)]
                assert sum(parts) % (1 << 64) == GOLD[name][f"P{k}"], (name, k)
    for seed in range(4):
        n = 30 + 20 * seed
        rp, col = csr_from_edges(n, random_graph(n, 0.2 + 0.1 * seed, 700 + seed))
        with DeviceGraph(rp, col) as d:
            for k in (7, 8):
                assert d.pattern_count(k) == orc.pattern(rp, col, k), (seed, k)


def test_clique_route_on_graphs_with_hubs(monkeypatch):
    """The route P7 and P8 take by themselves on graphs with a vertex above
    degree 4,096 (the graph with one vertex of degree 20,000), and forced on
    the Chung-Lu graph with hubs of degree 2,187, 1,525 and 1,173: both equal
    the counts the literal oracle committed, and the formula route agrees."""
    sys.path.insert(0, GOLDEN)
    from make_hub_golden import hub_graph
    with open(os.path.join(GOLDEN, "hub_counts.json")) as f:
        hub_want = json.load(f)["counts"]
    rp, col = hub_graph()
    with DeviceGraph(rp, col) as d:
        for k in (7, 8):
            assert d.pattern_count(k) == hub_want[f"P{k}"], k
            parts = [d.pattern_count_shard(k, s, 2) for s in range(2)]
            assert sum(parts) % (1 << 64) == hub_want[f"P{k}"], k
    monkeypatch.setenv("MERCURY_CLIQUE_ROUTE", "formula")
    with DeviceGraph(rp, col) as d:
        assert d.pattern_count(7) == hub_want["P7"]
    with open(os.path.join(GOLDEN, "pattern_counts.json")) as f:
        want = json.load(f)["chung_lu_n5000_mean20_cap50000_seed1"]["counts"]
    monkeypatch.setenv("MERCURY_CLIQUE_ROUTE", "cliques")
    g = Graph.chung_lu(5000, 2.1, 20.0, 50000.0, seed=1)
    with DeviceGraph(g) as d:
        for k in (7, 8):
            assert d.pattern_count(k) == want[f"P{k}"], k
            count, frac = d.pattern_count_budget(k, 60000.0)
            assert count == want[f"P{k}"] and frac == 1.0
