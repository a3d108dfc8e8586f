"""Set sizes that set the cost of the reference's pattern formulas, counted
on the CPU (tests/pattern_work.cpp): per directed edge (v0, v1), A = N(v0) &
N(v1) and B = N(v1) - N(v0).  The tests check the listing-based count against
sparse-matrix products on small graphs.  Run as a script, it prints the
figures for the pattern benchmark graph at a given size (default: Chung-Lu
n = 10^6, gamma 2.1, mean 20, cap 50,000, seed 1) that the design notes
quote:  python tests/test_pattern_work.py [n mean cap]
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FIELDS = ("triangles", "sum_d3", "sum_directed_A3", "directed_edges_A_over_32",
          "sum_directed_A_times_B", "sum_d2")
_lib = None


def lib():
    global _lib
    if _lib is None:
        out = os.path.join(HERE, "_build", "libpattern_work.so")
        src = os.path.join(HERE, "pattern_work.cpp")
        if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
            os.makedirs(os.path.dirname(out), exist_ok=True)
            subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", src,
                            "-o", out], check=True)
        _lib = C.CDLL(out)
    return _lib


def pattern_work(rowptr, col) -> dict:
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    ci = np.ascontiguousarray(col, dtype=np.int32)
    out = np.zeros(len(FIELDS))
    lib().pattern_work(C.c_int64(len(rp) - 1), C.c_void_p(rp.ctypes.data),
                       C.c_void_p(ci.ctypes.data), C.c_void_p(out.ctypes.data))
    return {k: float(v) for k, v in zip(FIELDS, out)}


@pytest.mark.parametrize("make", ["rmat", "chung_lu"])
def test_listing_count_equals_sparse_products(make):
    import scipy.sparse as sp
    from mercury_b200 import Graph
    g = Graph.rmat(11, 16, seed=4) if make == "rmat" else \
        Graph.chung_lu(3000, 2.1, 12.0, 400.0, seed=5)
    rp, col = np.asarray(g.rowptr), np.asarray(g.col)
    n = len(rp) - 1
    adj = sp.csr_matrix((np.ones(len(col)), col, rp), shape=(n, n))
    t = (adj @ adj).multiply(adj).tocsr()  # t[u, v] = |N(u) & N(v)| on edges
    deg = np.diff(rp).astype(np.float64)
    rows = np.repeat(np.arange(n), np.diff(t.indptr))
    a = t.data
    b = deg[t.indices] - a  # |N(v1) - N(v0)| for the directed edge (row, col)
    w = pattern_work(rp, col)
    assert w["triangles"] == a.sum() / 6
    assert w["sum_directed_A3"] == pytest.approx((a ** 3).sum(), rel=1e-12)
    # directed edges with no triangle are absent from t but add nothing
    assert w["directed_edges_A_over_32"] == (a > 32).sum()
    assert w["sum_directed_A_times_B"] == pytest.approx((a * b).sum(), rel=1e-12)
    assert w["sum_d3"] == (deg ** 3).sum() and w["sum_d2"] == (deg ** 2).sum()
    assert len(rows) == len(a)


if __name__ == "__main__":
    from mercury_b200 import Graph
    n, mean, cap = 1000000, 20.0, 50000.0
    if len(sys.argv) > 3:
        n, mean, cap = int(sys.argv[1]), float(sys.argv[2]), float(sys.argv[3])
    g = Graph.chung_lu(n, 2.1, mean, cap, seed=1)
    print(f"Chung-Lu n={n} gamma 2.1 mean {mean:g} cap {cap:g} seed 1: m = {g.nnz // 2:,}, "
          f"max degree {g.max_degree:,}")
    for k, v in pattern_work(g.rowptr, g.col).items():
        print(f"{k:28s} {v:.4g}")
