"""ORACLE -- test infrastructure, not product code.

ctypes loader of the CPU restatement in oracle/oracle.cpp and
oracle/patterns_oracle.cpp (built into oracle/_build/liboracle.so by
``make -C oracle``).  Only tests/, the smoke check and bench.py's CPU baseline
use it, always as the checker or the timed CPU baseline, never as a path of
the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_num_threads.restype = C.c_int
        L.orc_orient.argtypes = [C.c_int64, P, P, P, P]
        L.orc_orient.restype = None
        L.orc_division.argtypes = [C.c_int64, P, P, C.c_int, P]
        L.orc_division.restype = None
        L.orc_tc_dag.argtypes = [C.c_int64, P, P, C.c_int64, C.c_int64]
        L.orc_tc_dag.restype = C.c_uint64
        L.orc_tc_sample.argtypes = [C.c_int64, P, P, C.c_uint64, C.c_uint64, P]
        L.orc_tc_sample.restype = C.c_uint64
        L.orc_merge_volume.argtypes = [C.c_int64, P, P]
        L.orc_merge_volume.restype = C.c_double
        L.orc_tc.argtypes = [C.c_int64, P, P]
        L.orc_tc.restype = C.c_uint64
        L.orc_pattern.argtypes = [C.c_int64, P, P, C.c_int, P]
        L.orc_pattern.restype = C.c_uint64
        L.orc_tc_by_label.argtypes = [C.c_int64, P, P, P, C.c_int, P]
        L.orc_tc_by_label.restype = None
        L.orc_pattern_fast.argtypes = [C.c_int64, P, P, C.c_int, P]
        L.orc_pattern_fast.restype = C.c_uint64
        L.orc_clique_patterns.argtypes = [C.c_int64, P, P, P, P]
        L.orc_clique_patterns.restype = C.c_int
        L.orc_csr_build.argtypes = [C.c_int64, C.c_int64, P, P, P, P]
        L.orc_csr_build.restype = C.c_int64
        L.orc_rmat_draws.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_uint64, P, P]
        L.orc_rmat_draws.restype = C.c_int64
        L.orc_chung_lu_draws.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double,
                                         C.c_uint64, P, P]
        L.orc_chung_lu_draws.restype = C.c_int64
        _lib = L
    return _lib


def _csr(rowptr, col):
    return (np.ascontiguousarray(rowptr, dtype=np.int64),
            np.ascontiguousarray(col, dtype=np.int32))


def num_threads() -> int:
    return lib().orc_num_threads()


def orient(rowptr, col):
    """Degree-ordered DAG (graph.cc:196-235) as (dag_rowptr, dag_col)."""
    rowptr, col = _csr(rowptr, col)
    n = len(rowptr) - 1
    drp = np.zeros(n + 1, dtype=np.int64)
    lib().orc_orient(n, rowptr.ctypes.data, col.ctypes.data, drp.ctypes.data, None)
    dcol = np.zeros(max(int(drp[-1]), 1), dtype=np.int32)
    lib().orc_orient(n, rowptr.ctypes.data, col.ctypes.data, drp.ctypes.data, dcol.ctypes.data)
    return drp, dcol[: int(drp[-1])]


def division(rowptr, col, deg_thd: int = 128) -> dict:
    """Sizes of the reference's small/large split (graph.cc:237-312)."""
    rowptr, col = _csr(rowptr, col)
    out = np.zeros(4, dtype=np.int64)
    lib().orc_division(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data, deg_thd,
                       out.ctypes.data)
    return {"small_edges": int(out[0]), "large_edges": int(out[1]),
            "small_tasks": int(out[2]), "large_tasks": int(out[3])}


def tc(rowptr, col) -> int:
    rowptr, col = _csr(rowptr, col)
    return int(lib().orc_tc(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data))


def tc_by_label(rowptr, col, labels, max_label: int) -> np.ndarray:
    """Triangles split by the label of their DAG sink (labelled intersect_num)."""
    rowptr, col = _csr(rowptr, col)
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    out = np.zeros(max_label + 1, dtype=np.uint64)
    lib().orc_tc_by_label(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data,
                          labels.ctypes.data, max_label, out.ctypes.data)
    return out


def nlf(rowptr, col, labels, max_label: int) -> np.ndarray:
    """Dense neighbourhood label frequency (Graph::BuildNLF, numpy)."""
    rowptr, col = _csr(rowptr, col)
    labels = np.asarray(labels, dtype=np.int64)
    n = len(rowptr) - 1
    src = np.repeat(np.arange(n), np.diff(rowptr))
    out = np.zeros((n, max_label + 1), dtype=np.uint32)
    np.add.at(out, (src, labels[col]), 1)
    return out


def label_reverse_index(labels, max_label: int):
    """(offsets, vertices) of Graph::BuildReverseIndex (numpy, stable by id)."""
    labels = np.asarray(labels, dtype=np.int64)
    freq = np.bincount(labels, minlength=max_label + 1)
    off = np.zeros(max_label + 2, dtype=np.int64)
    np.cumsum(freq, out=off[1:])
    return off, np.argsort(labels, kind="stable").astype(np.int32)


def tc_dag(dag_rowptr, dag_col, v0: int = 0, v1: int | None = None) -> int:
    dag_rowptr, dag_col = _csr(dag_rowptr, dag_col)
    n = len(dag_rowptr) - 1
    return int(lib().orc_tc_dag(n, dag_rowptr.ctypes.data, dag_col.ctypes.data, v0,
                                n if v1 is None else v1))


def tc_sample(dag_rowptr, dag_col, modulus: int, seed: int = 0x5EED):
    """(count, DAG edges owned) over a hash-sampled 1/modulus of the sources."""
    dag_rowptr, dag_col = _csr(dag_rowptr, dag_col)
    edges = np.zeros(1, dtype=np.int64)
    c = lib().orc_tc_sample(len(dag_rowptr) - 1, dag_rowptr.ctypes.data, dag_col.ctypes.data,
                            modulus, seed, edges.ctypes.data)
    return int(c), int(edges[0])


def merge_volume(dag_rowptr, dag_col) -> float:
    dag_rowptr, dag_col = _csr(dag_rowptr, dag_col)
    return float(lib().orc_merge_volume(len(dag_rowptr) - 1, dag_rowptr.ctypes.data,
                                        dag_col.ctypes.data))


def pattern(rowptr, col, k: int, return_counters: bool = False):
    """Reference result of pattern P<k> (1..8)."""
    rowptr, col = _csr(rowptr, col)
    c12 = np.zeros(2, dtype=np.uint64)
    r = int(lib().orc_pattern(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data, k,
                              c12.ctypes.data))
    if return_counters:
        return r, int(c12[0]), int(c12[1])
    return r


def pattern_fast(rowptr, col, k: int, return_counters: bool = False):
    """P1 or P4 from the second restatement (patterns_fast.cpp: the same sets
    counted through position marks), for graphs whose hubs make pattern()
    take hours."""
    if k not in (1, 4):
        raise ValueError("pattern_fast restates P1 and P4 only")
    rowptr, col = _csr(rowptr, col)
    c12 = np.zeros(2, dtype=np.uint64)
    r = int(lib().orc_pattern_fast(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data, k,
                                   c12.ctypes.data))
    if return_counters:
        return r, int(c12[0]), int(c12[1])
    return r


def clique_patterns(rowptr, col, return_terms: bool = False):
    """{7: P7, 8: P8} from their clique restatement (clique_patterns.cpp:
    inclusion-exclusion over triangle, K4 and K5 counts), for graphs whose
    hubs make pattern() take days; None when the maximum degree exceeds
    46,340 (the reference's 32-bit products could wrap there)."""
    rowptr, col = _csr(rowptr, col)
    out = np.zeros(2, dtype=np.uint64)
    terms = np.zeros(7)
    rc = lib().orc_clique_patterns(len(rowptr) - 1, rowptr.ctypes.data, col.ctypes.data,
                                   out.ctypes.data, terms.ctypes.data)
    if rc != 0:
        return None
    counts = {7: int(out[0]), 8: int(out[1])}
    if return_terms:
        keys = ("triangles", "k4", "k5", "sum_c_a3", "sum_k4e_a2", "sum_3_c_k4t2", "ten_k5")
        return counts, {k: float(v) for k, v in zip(keys, terms)}
    return counts


def csr_from_edges(src, dst, n: int):
    """Symmetric CSR of the simple undirected graph on [0, n) given by the
    pairs (numpy restatement: the entry set of a networkx Graph built from
    the pairs, datasets/tsv2mtx.py:13, without self-loops, sorted)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if len(src) and (src.min() < 0 or dst.min() < 0 or src.max() >= n or dst.max() >= n):
        raise ValueError("id outside [0, n)")
    keep = src != dst
    u = np.concatenate([src[keep], dst[keep]])
    v = np.concatenate([dst[keep], src[keep]])
    key = np.unique(u * max(n, 1) + v)
    rows = key // max(n, 1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n)[:n], out=rowptr[1:])
    return rowptr, (key % max(n, 1)).astype(np.int32)


def csr_build(src, dst, n: int):
    """The same CSR from the C++/OpenMP restatement (parallel sort of packed
    keys); the CPU baseline of the device build."""
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    col = np.zeros(max(2 * len(src), 1), dtype=np.int32)
    nnz = lib().orc_csr_build(n, len(src), src.ctypes.data, dst.ctypes.data,
                              rowptr.ctypes.data, col.ctypes.data)
    if nnz < 0:
        raise ValueError("id outside [0, n)")
    return rowptr, col[:nnz]


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1):
    """Symmetric CSR (rowptr, col) of the seeded RMAT graph, built on the CPU
    (gen_oracle.cpp + csr_oracle.cpp) without the product library."""
    pairs = lib().orc_rmat_draws(scale, edge_factor, a, b, c, seed, None, None)
    if pairs < 0:
        raise ValueError("RMAT arguments outside the generator's range")
    src = np.empty(pairs, dtype=np.int32)
    dst = np.empty(pairs, dtype=np.int32)
    lib().orc_rmat_draws(scale, edge_factor, a, b, c, seed, src.ctypes.data, dst.ctypes.data)
    return csr_build(src, dst, 1 << scale)


def chung_lu(n: int, gamma: float = 2.1, mean_degree: float = 20.0, max_weight: float = 50000.0,
             seed: int = 1):
    """Symmetric CSR (rowptr, col) of the seeded Chung-Lu graph, built on the
    CPU without the product library."""
    pairs = lib().orc_chung_lu_draws(n, gamma, mean_degree, max_weight, seed, None, None)
    if pairs < 0:
        raise ValueError("Chung-Lu arguments outside the generator's range")
    src = np.empty(pairs, dtype=np.int32)
    dst = np.empty(pairs, dtype=np.int32)
    lib().orc_chung_lu_draws(n, gamma, mean_degree, max_weight, seed, src.ctypes.data,
                             dst.ctypes.data)
    return csr_build(src, dst, n)
