"""Edge lists and the device CSR build (the reference's dataset preparation).

The reference prepares its inputs offline: ``datasets/tsv2mtx.py`` turns a
GraphChallenge TSV into a Matrix Market file through a networkx ``Graph``
(undirected, duplicates merged), and the closed binary ``converter mtx
<file> <prefix> ...`` (``datasets/converter.sh:5``) writes the
graph.meta.txt / graph.vertex.bin / graph.edge.bin triple. Here the text is
parsed on the host (``EdgeList.load``), and the CSR is built on the GPU
(``EdgeList.to_graph`` / ``EdgeList.to_device``): symmetrise, drop
self-loops, merge duplicates, sort rows.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _ffi
from ._ffi import Timing, check, lib
from .graph import DeviceGraph, Graph

__all__ = ["EdgeList", "FORMATS"]

FORMATS = {"mtx": _ffi.MC_EDGES_MTX, "tsv": _ffi.MC_EDGES_TSV, "snap": _ffi.MC_EDGES_SNAP}


class EdgeList:
    """Host edge list (``mc_edges_t``): int32 endpoint pairs over [0, n)."""

    def __init__(self, *, _handle: int):
        self._h = C.c_void_p(_handle)
        self.last_timing = Timing()

    @classmethod
    def load(cls, path: str, fmt: str = "mtx", id_base: int = -1) -> "EdgeList":
        """Parses an "mtx", "tsv" or "snap" file; id_base -1 takes the format's
        default (1 for mtx and tsv, 0 for snap)."""
        h = C.c_void_p()
        check(lib().mc_edges_load(path.encode(), FORMATS[fmt], id_base, C.byref(h)),
              f"loading {path}")
        return cls(_handle=h.value)

    @classmethod
    def from_arrays(cls, src, dst, n: int) -> "EdgeList":
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        if src.shape != dst.shape:
            raise ValueError("src and dst differ in length")
        h = C.c_void_p()
        check(lib().mc_edges_from_arrays(src.ctypes.data if len(src) else None,
                                         dst.ctypes.data if len(dst) else None,
                                         len(src), n, C.byref(h)), "wrapping edge arrays")
        return cls(_handle=h.value)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1) -> "EdgeList":
        """The raw draws behind ``Graph.rmat`` with the same arguments."""
        h = C.c_void_p()
        check(lib().mc_gen_rmat_edges(scale, edge_factor, a, b, c, seed, C.byref(h)),
              "RMAT edge draws")
        return cls(_handle=h.value)

    @classmethod
    def chung_lu(cls, n: int, gamma: float = 2.1, mean_degree: float = 20.0,
                 max_weight: float = 50000.0, seed: int = 1) -> "EdgeList":
        """The raw draws behind ``Graph.chung_lu`` with the same arguments."""
        h = C.c_void_p()
        check(lib().mc_gen_chung_lu_edges(n, gamma, mean_degree, max_weight, seed, C.byref(h)),
              "Chung-Lu edge draws")
        return cls(_handle=h.value)

    def _info(self):
        m, n = C.c_int64(), C.c_int64()
        check(lib().mc_edges_info(self._h, C.byref(m), C.byref(n)), "edge list info")
        return m.value, n.value

    @property
    def num_edges(self) -> int:
        return self._info()[0]

    @property
    def n(self) -> int:
        return self._info()[1]

    def _view(self, fn) -> np.ndarray:
        m = self.num_edges
        if m == 0:
            return np.zeros(0, dtype=np.int32)
        arr = np.ctypeslib.as_array(C.cast(fn(self._h), C.POINTER(C.c_int32)), shape=(m,))
        arr.flags.writeable = False
        return arr

    @property
    def src(self) -> np.ndarray:
        return self._view(lib().mc_edges_src)

    @property
    def dst(self) -> np.ndarray:
        return self._view(lib().mc_edges_dst)

    def to_graph(self, n: Optional[int] = None, stream: Optional[int] = None) -> Graph:
        """Symmetric CSR built on the GPU, copied back as a host ``Graph``."""
        return csr_build(self.src, self.dst, self.n if n is None else n, stream=stream,
                         timing=self.last_timing)

    def to_device(self, n: Optional[int] = None, stream: Optional[int] = None,
                  validate_symmetry: bool = False) -> DeviceGraph:
        """Symmetric CSR built on the GPU and kept there as a ``DeviceGraph``."""
        return dgraph_from_edges(self.src, self.dst, self.n if n is None else n, stream=stream,
                                 validate_symmetry=validate_symmetry, timing=self.last_timing)

    def close(self) -> None:
        if self._h and self._h.value:
            lib().mc_edges_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pairs(src, dst, device: bool):
    if device:
        return int(src), int(dst), None
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    if src.shape != dst.shape:
        raise ValueError("src and dst differ in length")
    keep = (src, dst)
    return (src.ctypes.data if len(src) else None, dst.ctypes.data if len(dst) else None, keep)


def csr_build(src, dst, n: int, *, num_edges: Optional[int] = None, device_input: bool = False,
              stream: Optional[int] = None, timing: Optional[Timing] = None) -> Graph:
    """``mc_csr_build``: host (numpy) or device (pointer) pairs -> host Graph."""
    ps, pd, keep = _pairs(src, dst, device_input)
    m = num_edges if device_input else len(keep[0])
    flags = _ffi.MC_BUILD_DEVICE_INPUT if device_input else 0
    h = C.c_void_p()
    t = timing if timing is not None else Timing()
    check(lib().mc_csr_build(ps, pd, m, n, flags, stream, C.byref(h), C.byref(t)),
          "building the CSR on the device")
    return Graph(_handle=h.value)


def dgraph_from_edges(src, dst, n: int, *, num_edges: Optional[int] = None,
                      device_input: bool = False, stream: Optional[int] = None,
                      validate_symmetry: bool = False,
                      timing: Optional[Timing] = None) -> DeviceGraph:
    """``mc_dgraph_from_edges``: pairs -> device-resident DeviceGraph."""
    ps, pd, keep = _pairs(src, dst, device_input)
    m = num_edges if device_input else len(keep[0])
    flags = (_ffi.MC_BUILD_DEVICE_INPUT if device_input else 0) | (
        _ffi.MC_VALIDATE_SYMMETRY if validate_symmetry else 0)
    h = C.c_void_p()
    t = timing if timing is not None else Timing()
    check(lib().mc_dgraph_from_edges(ps, pd, m, n, flags, stream, C.byref(h), C.byref(t)),
          "building a device graph from edges")
    return DeviceGraph._adopt(h, n)
