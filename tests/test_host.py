"""Host logic behind the C ABI: file format, contract checks, generators."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mercury_b200 import Graph, McError
from mercury_b200 import _ffi


def fixture_prefix(name):
    return os.path.join(GOLDEN, "graphs", name, "graph")


@pytest.mark.parametrize("name", ["k5", "rmat10", "isolated", "dense400"])
def test_load_matches_files(name):
    p = fixture_prefix(name)
    g = Graph(p)
    assert np.array_equal(g.rowptr, np.fromfile(p + ".vertex.bin", dtype=np.int64))
    assert np.array_equal(g.col, np.fromfile(p + ".edge.bin", dtype=np.int32))
    g.validate(symmetry=True)


def test_write_then_load_round_trip(tmp_path):
    g = Graph.rmat(9, 8, seed=3)
    prefix = str(tmp_path / "graph")
    g.write(prefix)
    h = Graph(prefix)
    assert h.n == g.n and h.nnz == g.nnz and h.max_degree == g.max_degree
    assert np.array_equal(h.rowptr, g.rowptr) and np.array_equal(h.col, g.col)
    meta = open(prefix + ".meta.txt").read().split()
    assert len(meta) == 10 and meta[2:6] == ["4", "8", "1", "2"]


def _write(prefix, meta, rowptr, col):
    with open(prefix + ".meta.txt", "w") as f:
        f.write(meta)
    np.asarray(rowptr, dtype=np.int64).tofile(prefix + ".vertex.bin")
    np.asarray(col, dtype=np.int32).tofile(prefix + ".edge.bin")


def test_loader_errors(tmp_path):
    p = str(tmp_path / "g")
    rp, col = [0, 1, 2], [1, 0]
    with pytest.raises(McError) as e:
        Graph(str(tmp_path / "missing"))
    assert e.value.status == _ffi.MC_ERR_IO
    _write(p, "2 2 8 8 1 2 1 0 0 0", rp, col)  # vid_size 8: reference asserts 4
    with pytest.raises(McError) as e:
        Graph(p)
    assert e.value.status == _ffi.MC_ERR_FORMAT
    _write(p, "2 2 4 8 1 2 2 0 0 0", rp, col)  # max_degree must be < nv
    with pytest.raises(McError) as e:
        Graph(p)
    assert e.value.status == _ffi.MC_ERR_FORMAT
    _write(p, "2 4 4 8 1 2 1 0 0 0", rp, col)  # edge.bin shorter than ne
    with pytest.raises(McError) as e:
        Graph(p)
    assert e.value.status == _ffi.MC_ERR_FORMAT
    _write(p, "2 2 4 8 1 2 1 0 0 0", rp, col)
    assert Graph(p).nnz == 2


@pytest.mark.parametrize("rowptr,col", [
    ([0, 2, 3, 4], [2, 1, 0, 0]),      # unsorted row 0
    ([0, 2, 3, 4], [1, 1, 0, 0]),      # duplicate
    ([0, 2, 3, 5], [1, 2, 0, 0, 2]),   # self-loop at 2
    ([0, 1, 2], [1, 5]),               # id out of range
    ([0, 1, 1], [1]),                  # asymmetric
])
def test_validate_rejects(rowptr, col):
    g = Graph.from_csr(np.array(rowptr), np.array(col))
    with pytest.raises(McError) as e:
        g.validate(symmetry=True)
    assert e.value.status == _ffi.MC_ERR_FORMAT


def test_from_csr_rejects_bad_offsets():
    with pytest.raises(McError):
        Graph.from_csr(np.array([0, 2, 1]), np.array([1, 0]))


def test_rmat_is_deterministic_and_well_formed():
    a = Graph.rmat(12, 16, seed=1)
    b = Graph.rmat(12, 16, seed=1)
    c = Graph.rmat(12, 16, seed=2)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.rowptr, b.rowptr)
    assert not np.array_equal(a.col, c.col)
    a.validate(symmetry=True)
    assert a.n == 4096 and a.nnz % 2 == 0
    # skewed (a=0.57): vertex 0 is the largest hub
    assert int(np.argmax(np.diff(a.rowptr))) == 0


def test_chung_lu_stats():
    g = Graph.chung_lu(20000, gamma=2.1, mean_degree=20, max_weight=500, seed=4)
    g.validate(symmetry=True)
    mean = g.nnz / g.n
    assert 10 < mean <= 20
    assert g.max_degree <= 700
