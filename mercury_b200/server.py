"""Serving: counting requests with continuous batching (``mc_server_*`` in
include/mercury.h)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from ._ffi import McError, check, lib, MC_ERR_TIMEOUT
from .batch import job_code
from .graph import Graph


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in (
        "submitted", "completed", "failed", "batches", "cache_hits",
        "cache_bytes", "cached_graphs", "queued", "max_batch_seen")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Server:
    """Request loop on the current GPU with an HBM budget (bytes)."""

    def __init__(self, hbm_budget_bytes: int, max_batch: int = 1024, workers: int = 2):
        self._h = C.c_void_p()
        check(lib().mc_server_create(hbm_budget_bytes, max_batch, workers, C.byref(self._h)),
              "starting the server")

    def submit(self, graph=None, job="TC", key: int = 0) -> int:
        """Queues a request; `graph` may be None when `key` is resident."""
        if graph is None:
            rp = col = None
            n = nnz = 0
        else:
            if isinstance(graph, Graph):
                rp, col = np.asarray(graph.rowptr), np.asarray(graph.col)
            else:
                rp = np.ascontiguousarray(graph[0], dtype=np.int64)
                col = np.ascontiguousarray(graph[1], dtype=np.int32)
            n, nnz = len(rp) - 1, len(col)
        t = C.c_uint64()
        check(lib().mc_server_submit(self._h, None if rp is None else rp.ctypes.data,
                                     None if col is None or nnz == 0 else col.ctypes.data,
                                     n, nnz, job_code(job), key, C.byref(t)), "submitting")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000) -> Tuple[int, float]:
        """(count, latency in ms); raises McError (MC_ERR_TIMEOUT when late)."""
        c, lat = C.c_uint64(), C.c_double()
        check(lib().mc_server_wait(self._h, ticket, timeout_ms, C.byref(c), C.byref(lat)),
              f"request {ticket}")
        return c.value, lat.value

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().mc_server_stats(self._h, C.byref(st)), "server stats")
        return st.as_dict()

    def close(self) -> None:
        if self._h and self._h.value:
            lib().mc_server_free(self._h)
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
