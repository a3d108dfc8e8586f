"""P1..P8 on the GPU vs the golden fixtures, the reference programs' outputs
and the oracle (bit-exact uint64), through the C ABI."""
import json
import os

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


def test_patterns_chung_lu_vs_oracle():
    g = Graph.chung_lu(4000, 2.1, 10.0, 200.0, seed=9)
    rp, col = np.array(g.rowptr), np.array(g.col)
    with DeviceGraph(g) as d:
        for k in (1, 4, 6, 8):
            assert d.pattern_count(k) == orc.pattern(rp, col, k), k


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
