"""Batches: many graphs, each with its own job, counted in one captured
CUDA-graph launch (``mc_batch_*`` in include/mercury.h)."""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Sequence

import numpy as np

from ._ffi import Timing, check, lib
from .graph import Graph

JOBS = {"TC": 0, **{f"P{k}": k for k in range(1, 9)}}


def job_code(job) -> int:
    if isinstance(job, (int, np.integer)):
        if not 0 <= int(job) <= 8:
            raise ValueError(f"job {job} is not 0 (TC) or 1..8")
        return int(job)
    return JOBS[str(job).upper()]


def union_csr(graphs: Sequence):
    """Disjoint union of CSR graphs: (rowptr, col, graph_vptr)."""
    parts = []
    for g in graphs:
        if isinstance(g, Graph):
            parts.append((np.asarray(g.rowptr), np.asarray(g.col)))
        else:
            rp, col = g
            parts.append((np.asarray(rp, dtype=np.int64), np.asarray(col, dtype=np.int32)))
    ns = np.array([len(rp) - 1 for rp, _ in parts], dtype=np.int64)
    nnzs = np.array([len(col) for _, col in parts], dtype=np.int64)
    vptr = np.zeros(len(parts) + 1, dtype=np.int64)
    np.cumsum(ns, out=vptr[1:])
    eoff = np.zeros(len(parts) + 1, dtype=np.int64)
    np.cumsum(nnzs, out=eoff[1:])
    rowptr = np.empty(int(vptr[-1]) + 1, dtype=np.int64)
    col = np.empty(int(eoff[-1]), dtype=np.int32)
    for i, (rp, c) in enumerate(parts):
        rowptr[vptr[i]:vptr[i + 1]] = rp[:-1] + eoff[i]
        col[eoff[i]:eoff[i + 1]] = c + vptr[i]
    rowptr[-1] = eoff[-1]
    return rowptr, col, vptr


class Batch:
    """Graphs plus jobs ("TC", "P1".."P8" or 0..8), resident on the GPU."""

    def __init__(self, graphs: Sequence, jobs: Iterable, stream: Optional[int] = None):
        rowptr, col, vptr = union_csr(graphs)
        codes = np.array([job_code(j) for j in jobs], dtype=np.int32)
        if len(codes) != len(vptr) - 1:
            raise ValueError("one job per graph")
        self.num_graphs = len(codes)
        self.jobs = codes
        self._h = C.c_void_p()
        check(lib().mc_batch_create(rowptr.ctypes.data, col.ctypes.data if len(col) else None,
                                    len(rowptr) - 1, len(col), vptr.ctypes.data, self.num_graphs,
                                    codes.ctypes.data, stream, C.byref(self._h)),
              "creating the batch")
        self.last_timing = Timing()

    def autotune(self) -> np.ndarray:
        """Per degree bucket {warp/CTA threshold, log2 table slots per key}."""
        choice = np.full(8, -1, dtype=np.int32)
        check(lib().mc_batch_autotune(self._h, choice.ctypes.data), "autotuning the batch")
        return choice.reshape(4, 2)

    def count(self) -> np.ndarray:
        out = np.zeros(self.num_graphs, dtype=np.uint64)
        check(lib().mc_batch_count(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                   C.byref(self.last_timing)), "batch count")
        return out

    def close(self) -> None:
        if self._h and self._h.value:
            lib().mc_batch_free(self._h)
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
