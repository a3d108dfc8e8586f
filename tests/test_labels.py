"""Vertex labels: the reference's label file and label helpers
(graph.cc:37-58 reads graph.vlabel.bin; computeLabelsFrequency,
BuildReverseIndex, BuildNLF and the labelled Graph::intersect_num,
graph.cc:396-495), restated on the device and checked against the oracle's
restatements (oracle/oracle.cpp orc_tc_by_label, oracle/oracle.py nlf and
label_reverse_index) and against brute force."""
import itertools
import os

import numpy as np
import pytest

from brute import random_graph
from conftest import GOLDEN, csr_from_edges
from mercury_b200 import DeviceGraph, Graph, McError
from oracle import oracle as orc


def _labels(n, max_label, seed):
    return np.random.default_rng(seed).integers(0, max_label + 1, n).astype(np.uint8)


def test_label_file_round_trip_and_refusals(tmp_path):
    g = Graph(os.path.join(GOLDEN, "graphs", "petersen", "graph"))
    prefix = str(tmp_path / "graph")
    g.write(prefix)
    h = Graph(prefix)
    assert h.vlabels is None
    lab = _labels(g.n, 3, 1)
    lab.tofile(prefix + ".vlabel.bin")
    h.load_vlabels(prefix)
    assert np.array_equal(h.vlabels, lab)
    lab[:-1].tofile(prefix + ".vlabel.bin")  # one byte short
    with pytest.raises(McError):
        h.load_vlabels(prefix)
    os.remove(prefix + ".vlabel.bin")
    with pytest.raises(McError):
        h.load_vlabels(prefix)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_labelled_count_equals_brute_force(seed):
    n = 24
    edges = random_graph(n, 0.35, seed)
    rp, col = csr_from_edges(n, edges)
    lab = _labels(n, 3, seed)
    adj = [set(col[rp[v]:rp[v + 1]]) for v in range(n)]
    deg = [len(a) for a in adj]
    want = np.zeros(4, dtype=np.uint64)
    for a, b, c in itertools.combinations(range(n), 3):
        if b in adj[a] and c in adj[a] and c in adj[b]:
            # the DAG sink: the largest in the order (degree, id) -- every
            # DAG edge points from the lower end to the higher one
            sink = max((a, b, c), key=lambda v: (deg[v], v))
            want[lab[sink]] += 1
    got = orc.tc_by_label(rp, col, lab, 3)
    assert np.array_equal(got, want)
    assert int(got.sum()) == orc.tc(rp, col)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [lambda: Graph(os.path.join(GOLDEN, "graphs", "cl3000", "graph")),
                                  lambda: Graph(os.path.join(GOLDEN, "graphs", "dense400", "graph")),
                                  lambda: Graph.rmat(14, 16, seed=3)])
@pytest.mark.parametrize("max_label", [0, 4, 200])
def test_device_label_helpers_equal_the_oracle(make, max_label):
    g = make()
    rp, col = np.asarray(g.rowptr), np.asarray(g.col)
    lab = _labels(g.n, max_label, max_label + 7)
    with DeviceGraph(g) as d:
        d.set_vlabels(lab, max_label)
        assert np.array_equal(d.label_frequency(),
                              np.bincount(lab, minlength=max_label + 1).astype(np.uint64))
        off, verts = d.label_reverse_index()
        woff, wverts = orc.label_reverse_index(lab, max_label)
        assert np.array_equal(off, woff) and np.array_equal(verts, wverts)
        want_nlf = orc.nlf(rp, col, lab, max_label)
        assert np.array_equal(d.label_nlf(), want_nlf)
        lo, hi = g.n // 3, g.n // 2
        assert np.array_equal(d.label_nlf(lo, hi), want_nlf[lo:hi])
        by = d.tc_count_by_label()
        assert np.array_equal(by, orc.tc_by_label(rp, col, lab, max_label))
        assert int(by.sum()) == d.tc_count()


@pytest.mark.gpu
def test_labels_above_the_maximum_are_refused():
    g = Graph(os.path.join(GOLDEN, "graphs", "k5", "graph"))
    with DeviceGraph(g) as d:
        with pytest.raises(McError):
            d.set_vlabels(np.array([0, 1, 2, 3, 9], dtype=np.uint8), 3)
        d.set_vlabels(np.array([0, 1, 2, 3, 3], dtype=np.uint8), 3)
        assert list(d.label_frequency()) == [1, 1, 1, 2]
