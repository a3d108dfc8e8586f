"""Edge-list input and the CSR-build oracle, on the CPU (no GPU calls).

The fixtures in tests/golden/edges/ were produced by the reference's own
datasets/tsv2mtx.py (TSV -> networkx Graph -> Matrix Market). edges.json
holds the symmetric CSR that networkx describes, as a SHA-256 digest
(tests/golden/make_edge_golden.py).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, csr_from_edges
from mercury_b200 import EdgeList, Graph
from mercury_b200._ffi import McError, MC_ERR_ARG, MC_ERR_FORMAT, MC_ERR_IO, MC_ERR_UNSUPPORTED
from oracle import oracle as orc

EDGES = os.path.join(GOLDEN, "edges")
META = json.load(open(os.path.join(EDGES, "edges.json")))


def digest(rowptr, col):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, dtype="<i8").tobytes())
    h.update(np.ascontiguousarray(col, dtype="<i4").tobytes())
    return h.hexdigest()


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


# ---- oracle pins -----------------------------------------------------------

@pytest.mark.parametrize("name", sorted(META))
def test_oracle_matches_networkx_on_reference_converter_output(name):
    """Both oracle restatements reproduce the networkx graph of tsv2mtx.py."""
    e = EdgeList.load(os.path.join(EDGES, name + ".mtx"), "mtx")
    assert e.n == META[name]["n"]
    # networkx merged the duplicate lines: the MTX lists each undirected edge
    # (self-loops included) once.
    assert META[name]["nnz"] // 2 <= e.num_edges < META[name]["lines"]
    a = orc.csr_from_edges(e.src, e.dst, e.n)
    b = orc.csr_build(e.src, e.dst, e.n)
    assert digest(*a) == META[name]["csr_sha256"]
    assert digest(*b) == META[name]["csr_sha256"]
    assert len(a[1]) == META[name]["nnz"]


@pytest.mark.parametrize("name", sorted(META))
def test_tsv_and_reference_mtx_give_the_same_graph(name):
    t = EdgeList.load(os.path.join(EDGES, name + ".tsv"), "tsv")
    m = EdgeList.load(os.path.join(EDGES, name + ".mtx"), "mtx")
    assert t.n == m.n == META[name]["n"]
    assert t.num_edges == META[name]["lines"]
    assert digest(*orc.csr_from_edges(t.src, t.dst, t.n)) == META[name]["csr_sha256"]


def test_oracle_matches_set_construction_on_random_pairs():
    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 64, 300):
        m = int(rng.integers(0, 4 * n + 1))
        s = rng.integers(0, n, m)
        d = rng.integers(0, n, m)
        want = csr_from_edges(n, list(zip(s.tolist(), d.tolist())))
        for got in (orc.csr_from_edges(s, d, n), orc.csr_build(s, d, n)):
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_generator_draws_build_the_generated_graph():
    """mc_gen_rmat_edges are the draws behind mc_gen_rmat (same seed)."""
    e = EdgeList.rmat(10, 8, seed=3)
    g = Graph.rmat(10, 8, seed=3)
    rp, col = orc.csr_from_edges(e.src, e.dst, e.n)
    assert np.array_equal(rp, g.rowptr) and np.array_equal(col, g.col)
    e = EdgeList.chung_lu(3000, seed=4)
    g = Graph.chung_lu(3000, seed=4)
    rp, col = orc.csr_from_edges(e.src, e.dst, e.n)
    assert np.array_equal(rp, g.rowptr) and np.array_equal(col, g.col)


# ---- parser -----------------------------------------------------------------

def test_mtx_header_comments_values_and_crlf(tmp_path):
    p = write(tmp_path, "a.mtx",
              "%%MatrixMarket matrix coordinate real general\r\n"
              "% a comment\r\n"
              "\r\n"
              "5 5 4\r\n"
              "1 2 0.5\r\n"
              "% inside the body\r\n"
              "2 3 1e3\r\n"
              "  4\t5\r\n"
              "5 5 2\r\n")
    e = EdgeList.load(p, "mtx")
    assert e.n == 5 and e.num_edges == 4
    assert e.src.tolist() == [0, 1, 3, 4] and e.dst.tolist() == [1, 2, 4, 4]


def test_mtx_vertex_count_covers_ids_beyond_the_size_line(tmp_path):
    # networkx writes the node count, which can be below the largest id.
    p = write(tmp_path, "b.mtx", "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n1 9\n9 4\n")
    e = EdgeList.load(p, "mtx")
    assert e.n == 9


def test_vidfrom0_base(tmp_path):
    p = write(tmp_path, "c.mtx", "%%MatrixMarket matrix coordinate pattern general\n3 3 2\n0 1\n1 2\n")
    with pytest.raises(McError) as ex:
        EdgeList.load(p, "mtx")  # 1-based by default: id 0 is invalid
    assert ex.value.status == MC_ERR_FORMAT
    e = EdgeList.load(p, "mtx", id_base=0)
    assert e.n == 3 and e.src.tolist() == [0, 1] and e.dst.tolist() == [1, 2]


def test_snap_and_tsv_defaults(tmp_path):
    s = EdgeList.load(write(tmp_path, "g.txt", "# SNAP\n# Nodes: 3\n0 1\n1\t2\n\n2 0\n"), "snap")
    assert s.n == 3 and s.num_edges == 3 and s.src.tolist() == [0, 1, 2]
    t = EdgeList.load(write(tmp_path, "g.tsv", "1\t2\t1\n2\t3\t1\n"), "tsv")
    assert t.n == 3 and t.src.tolist() == [0, 1] and t.dst.tolist() == [1, 2]


def test_empty_lists(tmp_path):
    e = EdgeList.load(write(tmp_path, "e.tsv", ""), "tsv")
    assert e.n == 0 and e.num_edges == 0
    e = EdgeList.load(write(tmp_path, "e.mtx", "%%MatrixMarket matrix coordinate pattern general\n4 4 0\n"), "mtx")
    assert e.n == 4 and e.num_edges == 0


@pytest.mark.parametrize("body,status", [
    ("1\n", MC_ERR_FORMAT),            # one field
    ("1 -2\n", MC_ERR_FORMAT),         # negative id
    ("1.5 2\n", MC_ERR_FORMAT),        # not an integer
    ("x y\n", MC_ERR_FORMAT),
    ("1 4294967297\n", MC_ERR_UNSUPPORTED),  # beyond int32 ids
    ("1 4611686018427387904\n", MC_ERR_UNSUPPORTED),  # 2^62: a number, beyond int32 ids
    ("1 4611686018427387905\n", MC_ERR_FORMAT),       # above 2^62: not read as a number
    ("1 9999999999999999999\n", MC_ERR_FORMAT),       # 19 digits: x * 10 would pass 2^63
    ("1 99999999999999999999\n", MC_ERR_FORMAT),      # 20 digits
])
def test_bad_lines_are_refused(tmp_path, body, status):
    with pytest.raises(McError) as ex:
        EdgeList.load(write(tmp_path, "bad.tsv", "1 2\n" + body), "tsv")
    assert ex.value.status == status


@pytest.mark.parametrize("text,status", [
    ("3 3 1\n1 2\n", MC_ERR_FORMAT),                                               # no banner
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", MC_ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 2\n2 3\n", MC_ERR_FORMAT),  # truncated
    ("%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 2\n2 3\n", MC_ERR_FORMAT),  # extra
    ("%%MatrixMarket matrix coordinate pattern general\n% no size line\n", MC_ERR_FORMAT),
    ("", MC_ERR_FORMAT),
])
def test_bad_mtx_files_are_refused(tmp_path, text, status):
    with pytest.raises(McError) as ex:
        EdgeList.load(write(tmp_path, "bad.mtx", text), "mtx")
    assert ex.value.status == status


def test_missing_file_and_bad_format(tmp_path):
    with pytest.raises(McError) as ex:
        EdgeList.load(str(tmp_path / "nope.mtx"), "mtx")
    assert ex.value.status == MC_ERR_IO
    from mercury_b200 import _ffi
    import ctypes as C
    h = C.c_void_p()
    assert _ffi.lib().mc_edges_load(str(tmp_path / "x").encode(), 9, -1, C.byref(h)) == MC_ERR_ARG


def test_large_file_is_parsed_by_several_threads_in_order(tmp_path):
    """A multi-megabyte file is split into chunks at line boundaries; the
    concatenation keeps file order."""
    rng = np.random.default_rng(11)
    m = 400_000
    s = rng.integers(1, 2_000_000, m)
    d = rng.integers(1, 2_000_000, m)
    lines = [f"{a}\t{b}\t1" for a, b in zip(s, d)]
    lines.insert(1000, "")
    p = write(tmp_path, "big.tsv", "\n".join(lines) + "\n")
    assert os.path.getsize(p) > (1 << 20)
    e = EdgeList.load(p, "tsv")
    assert e.num_edges == m
    assert np.array_equal(e.src, s - 1) and np.array_equal(e.dst, d - 1)
    assert e.n == int(max(s.max(), d.max()))


def test_from_arrays_round_trip():
    e = EdgeList.from_arrays([0, 3, 2], [1, 1, 2], 5)
    assert e.n == 5 and e.src.tolist() == [0, 3, 2] and e.dst.tolist() == [1, 1, 2]
    with pytest.raises(ValueError):
        EdgeList.from_arrays([0, 1], [1], 3)
