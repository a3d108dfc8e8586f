"""Host-side mirror of the reference's counting interface over the C ABI.

Reference names kept: ``Graph(prefix)`` loads the graph.meta.txt /
graph.vertex.bin / graph.edge.bin triple (graph.cc:6-35); ``TCSolver(g)``
returns the triangle count that ``void TCSolver(Graph&, uint64_t&)``
(tc_challenge.cu:11) writes; ``SMSolver(g, "P1".."P8")`` returns the count
``SMSolverMultiGPU`` (subgraph_matching/sm_multigpu.cu:97) prints, on one GPU
and without MPI.  Every count comes from the CUDA kernels behind
include/mercury.h; a failing call raises ``McError``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _ffi
from ._ffi import McError, Timing, TcStats, check, lib

__all__ = ["Graph", "DeviceGraph", "TCSolver", "tc_count_host", "McError", "Timing"]


def _as_csr(rowptr, col) -> Tuple[np.ndarray, np.ndarray]:
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    return rowptr, col


class Graph:
    """Host CSR graph (``mc_graph_t``): loaded, generated or wrapped."""

    def __init__(self, prefix: Optional[str] = None, *, _handle: Optional[int] = None):
        self._h = C.c_void_p()
        if _handle is not None:
            self._h = C.c_void_p(_handle)
        elif prefix is not None:
            check(lib().mc_graph_load(prefix.encode(), C.byref(self._h)), f"loading {prefix}")
        else:
            raise ValueError("Graph needs a file prefix (or use a constructor classmethod)")

    # -- constructors -----------------------------------------------------
    @classmethod
    def _adopt(cls, h: C.c_void_p) -> "Graph":
        return cls(_handle=h.value)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1) -> "Graph":
        h = C.c_void_p()
        check(lib().mc_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)), "RMAT generator")
        return cls._adopt(h)

    @classmethod
    def chung_lu(cls, n: int, gamma: float = 2.1, mean_degree: float = 20.0,
                 max_weight: float = 50000.0, seed: int = 1) -> "Graph":
        h = C.c_void_p()
        check(lib().mc_gen_chung_lu(n, gamma, mean_degree, max_weight, seed, C.byref(h)),
              "Chung-Lu generator")
        return cls._adopt(h)

    @classmethod
    def from_csr(cls, rowptr, col) -> "Graph":
        rowptr, col = _as_csr(rowptr, col)
        h = C.c_void_p()
        check(lib().mc_graph_from_csr(rowptr.ctypes.data, col.ctypes.data, len(rowptr) - 1,
                                      len(col), C.byref(h)), "wrapping CSR arrays")
        return cls._adopt(h)

    # -- accessors --------------------------------------------------------
    def _info(self):
        n, nnz, md = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mc_graph_info(self._h, C.byref(n), C.byref(nnz), C.byref(md)), "graph info")
        return n.value, nnz.value, md.value

    @property
    def n(self) -> int:
        return self._info()[0]

    @property
    def nnz(self) -> int:
        return self._info()[1]

    @property
    def max_degree(self) -> int:
        return self._info()[2]

    @property
    def rowptr(self) -> np.ndarray:
        """int64[n+1] view into the handle's memory (valid while self lives)."""
        n = self.n
        p = lib().mc_graph_rowptr(self._h)
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int64)), shape=(n + 1,))
        arr.flags.writeable = False
        return arr

    @property
    def col(self) -> np.ndarray:
        nnz = self.nnz
        if nnz == 0:
            return np.zeros(0, dtype=np.int32)
        p = lib().mc_graph_col(self._h)
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int32)), shape=(nnz,))
        arr.flags.writeable = False
        return arr

    def load_vlabels(self, prefix: str) -> None:
        """Reads <prefix>.vlabel.bin (one uint8 per vertex, graph.cc:37-58)."""
        check(lib().mc_graph_load_vlabels(self._h, prefix.encode()), f"labels of {prefix}")

    @property
    def vlabels(self) -> Optional[np.ndarray]:
        p = C.c_void_p()
        check(lib().mc_graph_vlabels(self._h, C.byref(p)), "graph labels")
        if not p.value:
            return None
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(self.n,)).copy()

    def validate(self, symmetry: bool = True) -> None:
        check(lib().mc_graph_validate(self._h, 1 if symmetry else 0), "graph contract")

    def write(self, prefix: str) -> None:
        check(lib().mc_graph_write(self._h, prefix.encode()), f"writing {prefix}")

    def close(self) -> None:
        if self._h and self._h.value:
            lib().mc_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceGraph:
    """Device-resident symmetric CSR (``mc_dgraph_t``) on the current GPU."""

    def __init__(self, rowptr, col=None, *, stream: Optional[int] = None,
                 validate_symmetry: bool = False, host_columns: bool = False,
                 host_dag: bool = False):
        """host_columns=True keeps the column array in pinned host memory that
        the kernels read through the device's mapping (MC_HOST_COLUMNS); the
        library also chooses it when the device cannot hold the graph.
        host_dag=True keeps the degree-ordered DAG there as well
        (MC_HOST_DAG), chosen by itself when even that does not fit."""
        if isinstance(rowptr, Graph):
            g = rowptr
            rowptr, col = g.rowptr, g.col
        rowptr, col = _as_csr(rowptr, col)
        self.n = len(rowptr) - 1
        self.nnz = len(col)
        self._h = C.c_void_p()
        flags = _ffi.MC_VALIDATE_SYMMETRY if validate_symmetry else 0
        if host_columns:
            flags |= _ffi.MC_HOST_COLUMNS
        if host_dag:
            flags |= _ffi.MC_HOST_DAG
        check(lib().mc_dgraph_create(rowptr.ctypes.data, col.ctypes.data if self.nnz else None,
                                     self.n, self.nnz, stream, flags, C.byref(self._h)),
              "uploading the graph")
        self.last_timing = Timing()

    @classmethod
    def from_device(cls, d_rowptr_ptr: int, d_col_ptr: int, n: int, nnz: int,
                    stream: Optional[int] = None, validate_symmetry: bool = False,
                    host_columns: bool = False) -> "DeviceGraph":
        """From a CSR already in device memory (e.g. torch tensors' data_ptr())."""
        self = cls.__new__(cls)
        self.n, self.nnz = n, nnz
        self._h = C.c_void_p()
        flags = _ffi.MC_VALIDATE_SYMMETRY if validate_symmetry else 0
        if host_columns:
            flags |= _ffi.MC_HOST_COLUMNS
        check(lib().mc_dgraph_create_device(d_rowptr_ptr, d_col_ptr, n, nnz, stream, flags,
                                            C.byref(self._h)), "adopting a device CSR")
        self.last_timing = Timing()
        return self

    @classmethod
    def _adopt(cls, h: C.c_void_p, n: int) -> "DeviceGraph":
        self = cls.__new__(cls)
        self._h = h
        self.last_timing = Timing()
        nn, nnz, md = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mc_dgraph_info(h, C.byref(nn), C.byref(nnz), C.byref(md)), "device graph info")
        self.n, self.nnz, self.max_degree = nn.value, nnz.value, md.value
        return self

    def export_csr(self) -> Tuple[np.ndarray, np.ndarray]:
        """The handle's symmetric CSR as host (rowptr, col)."""
        rp = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(max(self.nnz, 1), dtype=np.int32)
        check(lib().mc_dgraph_export_csr(self._h, rp.ctypes.data, col.ctypes.data), "export csr")
        return rp, col[: self.nnz]

    @property
    def columns_on_host(self) -> bool:
        """True when the column array lives in host memory (asked for, or
        chosen because the device could not hold the graph)."""
        v = C.c_int()
        check(lib().mc_dgraph_columns_on_host(self._h, C.byref(v)), "column placement")
        return bool(v.value)

    @property
    def dag_on_host(self) -> bool:
        """True when the DAG lives in host memory (MC_HOST_DAG, asked for or chosen)."""
        v = C.c_int()
        check(lib().mc_dgraph_dag_on_host(self._h, C.byref(v)), "DAG placement")
        return bool(v.value)

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().mc_dgraph_stream(self._h, C.byref(s)), "stream")
        return s.value or 0

    def tc_count(self) -> int:
        out = C.c_uint64()
        check(lib().mc_tc_count(self._h, C.byref(out), C.byref(self.last_timing)), "triangle count")
        return out.value

    def tc_count_shard(self, shard: int, num_shards: int) -> int:
        """Partial count of one shard (partials of all shards sum to tc_count)."""
        out = C.c_uint64()
        check(lib().mc_tc_count_shard(self._h, shard, num_shards, C.byref(out),
                                      C.byref(self.last_timing)), "sharded triangle count")
        return out.value

    def pattern_count(self, pattern) -> int:
        """Count of pattern P1..P8 (int 1..8 or the string "P1".."P8")."""
        k = int(str(pattern).upper().lstrip("P"))
        out = C.c_uint64()
        check(lib().mc_pattern_count(self._h, k, C.byref(out), C.byref(self.last_timing)),
              f"pattern P{k}")
        return out.value

    def pattern_count_budget(self, pattern, budget_ms: float):
        """(count, 1.0) within budget_ms of device time, or (None, fraction of
        the tasks done) when the budget ran out (mc_pattern_count_budget)."""
        k = int(str(pattern).upper().lstrip("P"))
        out = C.c_uint64()
        prog = C.c_double(0.0)
        rc = lib().mc_pattern_count_budget(self._h, k, float(budget_ms), C.byref(out),
                                           C.byref(prog), C.byref(self.last_timing))
        if rc == _ffi.MC_ERR_TIMEOUT:
            return None, prog.value
        check(rc, f"pattern P{k} (budget)")
        return out.value, prog.value

    def pattern_count_shard(self, pattern, shard: int, num_shards: int) -> int:
        """Partial count of one shard (partials of all shards sum to the count mod 2^64)."""
        k = int(str(pattern).upper().lstrip("P"))
        out = C.c_uint64()
        check(lib().mc_pattern_count_shard(self._h, k, shard, num_shards, C.byref(out),
                                           C.byref(self.last_timing)), f"pattern P{k} shard")
        return out.value

    def tc_stats(self) -> dict:
        st = TcStats()
        check(lib().mc_tc_stats(self._h, C.byref(st)), "tc stats")
        return st.as_dict()

    def export_dag(self) -> Tuple[np.ndarray, np.ndarray]:
        """Device-built DAG (after tc_count) as host (rowptr, col)."""
        rp = np.zeros(self.n + 1, dtype=np.int64)
        check(lib().mc_dgraph_export_dag(self._h, rp.ctypes.data, None), "export dag offsets")
        col = np.zeros(max(int(rp[-1]), 1), dtype=np.int32)
        check(lib().mc_dgraph_export_dag(self._h, rp.ctypes.data, col.ctypes.data), "export dag")
        return rp, col[: int(rp[-1])]

    # -- vertex labels (graph.cc:37-58, :396-495) -------------------------
    def set_vlabels(self, labels, max_label: int) -> None:
        """Copies one uint8 label per vertex to the device (labels <= max_label)."""
        labels = np.ascontiguousarray(labels, dtype=np.uint8)
        if len(labels) != self.n:
            raise ValueError("one label per vertex")
        self._max_label = int(max_label)
        check(lib().mc_dgraph_set_vlabels(self._h, labels.ctypes.data, int(max_label)),
              "vertex labels")

    def label_frequency(self) -> np.ndarray:
        """Vertices per label 0..max_label (computeLabelsFrequency)."""
        out = np.zeros(self._max_label + 1, dtype=np.uint64)
        check(lib().mc_label_frequency(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64))),
              "label frequency")
        return out

    def label_reverse_index(self) -> Tuple[np.ndarray, np.ndarray]:
        """(offsets, vertices): vertices grouped by label in id order
        (BuildReverseIndex / getVerticesByLabel)."""
        off = np.zeros(self._max_label + 2, dtype=np.int64)
        verts = np.zeros(max(self.n, 1), dtype=np.int32)
        check(lib().mc_label_reverse_index(self._h, off.ctypes.data, verts.ctypes.data),
              "label reverse index")
        return off, verts[: self.n]

    def label_nlf(self, v_begin: int = 0, v_end: Optional[int] = None) -> np.ndarray:
        """Rows of neighbour-label counts for vertices [v_begin, v_end) (BuildNLF)."""
        v_end = self.n if v_end is None else v_end
        out = np.zeros((max(v_end - v_begin, 0), self._max_label + 1), dtype=np.uint32)
        check(lib().mc_label_nlf(self._h, v_begin, v_end, out.ctypes.data if out.size else None),
              "neighbourhood label frequency")
        return out

    def tc_count_by_label(self) -> np.ndarray:
        """Triangles split by the label of their DAG sink (intersect_num with a
        label over the degree-ordered DAG); the entries sum to tc_count()."""
        out = np.zeros(self._max_label + 1, dtype=np.uint64)
        check(lib().mc_tc_count_by_label(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                         C.byref(self.last_timing)), "labelled triangle count")
        return out

    def close(self) -> None:
        if self._h and self._h.value:
            lib().mc_dgraph_free(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tc_count_host(rowptr, col, timing: Optional[Timing] = None) -> int:
    """One-shot count from host arrays (upload, orient, count, copy back)."""
    rowptr, col = _as_csr(rowptr, col)
    out = C.c_uint64()
    t = timing if timing is not None else Timing()
    check(lib().mc_tc_count_host(rowptr.ctypes.data, col.ctypes.data if len(col) else None,
                                 len(rowptr) - 1, len(col), C.byref(out), C.byref(t)),
          "one-shot triangle count")
    return out.value


def TCSolver(g: Graph) -> int:
    """Triangle count of a host graph, as the reference's TCSolver computes it."""
    return tc_count_host(g.rowptr, g.col)
