"""The oracle pinned against brute force and the golden fixtures (CPU only)."""
import json
import os

import numpy as np
import pytest

from brute import expected_from_counts, induced_counts, random_graph, triangles
from conftest import GOLDEN, csr_from_edges, relabel
from oracle import oracle as orc

with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)

CHEAP = ["k5", "star9", "path6", "petersen", "rand13", "isolated", "rmat8"]


def load_fixture(name):
    prefix = os.path.join(GOLDEN, "graphs", name, "graph")
    rp = np.fromfile(prefix + ".vertex.bin", dtype=np.int64)
    col = np.fromfile(prefix + ".edge.bin", dtype=np.int32)
    return rp, col


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_tc_matches_golden(name):
    rp, col = load_fixture(name)
    assert orc.tc(rp, col) == GOLD[name]["TC"]


@pytest.mark.parametrize("name", CHEAP)
def test_oracle_patterns_match_golden(name):
    rp, col = load_fixture(name)
    for k in range(1, 9):
        assert orc.pattern(rp, col, k) == GOLD[name][f"P{k}"], (name, k)


@pytest.mark.parametrize("seed", [101, 202, 303])
def test_oracle_formulas_are_the_induced_identities(seed):
    n = 12
    rp, col = csr_from_edges(n, random_graph(n, 0.4, seed))
    exp = expected_from_counts(induced_counts(rp, col))
    got = {"TC": orc.tc(rp, col), **{f"P{k}": orc.pattern(rp, col, k) for k in range(1, 9)}}
    assert got == exp


def test_oracle_tc_brute_force_rmat10():
    rp, col = load_fixture("rmat10")
    assert orc.tc(rp, col) == triangles(rp, col)


def test_relabel_invariance_of_oracle():
    rp, col = load_fixture("rmat8")
    perm = np.random.default_rng(5).permutation(len(rp) - 1)
    rp2, col2 = relabel(rp, col, perm)
    assert orc.tc(rp2, col2) == orc.tc(rp, col)
    # Pattern counts are induced-subgraph counts, so invariant too.
    for k in (1, 4, 6):
        assert orc.pattern(rp2, col2, k) == orc.pattern(rp, col, k)


def test_orientation_is_a_dag_with_every_edge_once():
    rp, col = load_fixture("cl3000")
    drp, dcol = orc.orient(rp, col)
    n = len(rp) - 1
    deg = np.diff(rp)
    assert drp[-1] * 2 == len(col)
    src = np.repeat(np.arange(n), np.diff(drp))
    key_s = deg[src] * (n + 1) + src
    key_d = deg[dcol] * (n + 1) + dcol
    assert np.all(key_d > key_s)  # strictly up the (degree, id) order
    for v in range(n):
        row = dcol[drp[v]:drp[v + 1]]
        assert np.all(np.diff(row) > 0)


def test_division_sizes_cover_the_contributing_edges():
    rp, col = load_fixture("dense400")
    d = orc.division(rp, col)
    drp, _ = orc.orient(rp, col)
    # dense400 has every out-degree >= 1 except the top vertex; every DAG
    # edge lands in exactly one of the two lists unless an end has d+ == 0.
    assert d["small_edges"] + d["large_edges"] <= drp[-1]
    assert d["large_edges"] > 0
    assert d == GOLD["dense400"]["division"]


@pytest.mark.parametrize("scale,ef,seed", [(8, 8, 3), (12, 16, 1), (14, 32, 7)])
def test_rmat_restatement_equals_library_generator(scale, ef, seed):
    from mercury_b200 import Graph
    rp, col = orc.rmat(scale, ef, seed=seed)
    g = Graph.rmat(scale, ef, seed=seed)
    assert np.array_equal(rp, g.rowptr) and np.array_equal(col, g.col)


@pytest.mark.parametrize("n,mean,cap,seed", [(5000, 10.0, 200.0, 1), (30000, 20.0, 5000.0, 2)])
def test_chung_lu_restatement_equals_library_generator(n, mean, cap, seed):
    from mercury_b200 import Graph
    rp, col = orc.chung_lu(n, 2.1, mean, cap, seed=seed)
    g = Graph.chung_lu(n, 2.1, mean, cap, seed=seed)
    assert np.array_equal(rp, g.rowptr) and np.array_equal(col, g.col)


@pytest.mark.parametrize("seed", range(5))
def test_fast_p1_p4_restatement_equals_literal_oracle(seed):
    """patterns_fast.cpp counts P1 and P4 through position marks; its counters
    c1 and c2 equal the literal restatement's on random graphs, the golden
    fixtures and a Chung-Lu graph with hubs."""
    n = 30 + 25 * seed
    rp, col = csr_from_edges(n, random_graph(n, 0.15 + 0.07 * seed, 100 + seed))
    for k in (1, 4):
        assert orc.pattern_fast(rp, col, k, True) == orc.pattern(rp, col, k, True), k


def test_fast_p1_p4_restatement_on_fixtures_and_hubs():
    for name in ("cl3000", "rmat10", "petersen", "isolated", "dense400"):
        prefix = os.path.join(GOLDEN, "graphs", name, "graph")
        rp = np.fromfile(prefix + ".vertex.bin", dtype=np.int64)
        col = np.fromfile(prefix + ".edge.bin", dtype=np.int32)
        for k in (1, 4):
            assert orc.pattern_fast(rp, col, k, True) == orc.pattern(rp, col, k, True), (name, k)
    rp, col = orc.chung_lu(20000, 2.1, 12.0, 2000.0, seed=4)
    for k in (1, 4):
        assert orc.pattern_fast(rp, col, k, True) == orc.pattern(rp, col, k, True), k


@pytest.mark.parametrize("seed", range(6))
def test_clique_restatement_equals_literal_oracle(seed):
    """clique_patterns.cpp counts P7 and P8 as inclusion-exclusion over
    triangle, K4 and K5 counts; both equal the literal restatement on random
    graphs of rising density."""
    n = 20 + 12 * seed
    rp, col = csr_from_edges(n, random_graph(n, 0.12 + 0.08 * seed, 400 + seed))
    c = orc.clique_patterns(rp, col)
    assert c[7] == orc.pattern(rp, col, 7) and c[8] == orc.pattern(rp, col, 8)


def test_clique_restatement_on_fixtures_and_hubs():
    """The golden fixtures, the Chung-Lu graph with hubs of degree 2,187,
    1,525 and 1,173 and the graph with a vertex of degree 20,000, whose P7 and
    P8 the literal oracle committed."""
    named = [name for name in sorted(GOLD) if "P7" in GOLD[name]]
    assert len(named) >= 5
    for name in named:
        rp, col = load_fixture(name)
        c = orc.clique_patterns(rp, col)
        assert (c[7], c[8]) == (GOLD[name]["P7"], GOLD[name]["P8"]), name
    with open(os.path.join(GOLDEN, "pattern_counts.json")) as f:
        rec = json.load(f)["chung_lu_n5000_mean20_cap50000_seed1"]
    rp, col = orc.chung_lu(5000, 2.1, 20.0, 50000.0, seed=1)
    c = orc.clique_patterns(rp, col)
    assert (c[7], c[8]) == (rec["counts"]["P7"], rec["counts"]["P8"])
    import sys
    sys.path.insert(0, GOLDEN)
    from make_hub_golden import hub_graph
    with open(os.path.join(GOLDEN, "hub_counts.json")) as f:
        hub = json.load(f)["counts"]
    c = orc.clique_patterns(*hub_graph())
    assert (c[7], c[8]) == (hub["P7"], hub["P8"])


def test_clique_restatement_refuses_degrees_where_products_wrap():
    """Above degree 46,340 the reference's 32-bit products can wrap and the
    identity no longer holds: the restatement refuses (None)."""
    n = 46342
    rp, col = csr_from_edges(n, [(0, v) for v in range(1, n)])
    assert orc.clique_patterns(rp, col) is None
