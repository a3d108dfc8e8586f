"""ctypes binding of the C ABI declared in include/mercury.h.

The shared library is built in-tree (mercury_b200/lib/libmercury_b200.so) by
``mercury_b200.build.build()``.  Loading fails loudly when it is missing:
there is no CPU fallback for any counting call.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libmercury_b200.so")

MC_OK = 0
MC_ERR_ARG = -1
MC_ERR_IO = -2
MC_ERR_FORMAT = -3
MC_ERR_OOM = -4
MC_ERR_CUDA = -5
MC_ERR_DEVICE = -6
MC_ERR_UNSUPPORTED = -7
MC_ERR_NO_DEVICE = -8
MC_ERR_BUDGET = -9
MC_ERR_TIMEOUT = -10

MC_VALIDATE_SYMMETRY = 0x1
MC_HOST_COLUMNS = 0x2
MC_HOST_DAG = 0x4
MC_BUILD_DEVICE_INPUT = 0x100

MC_EDGES_MTX = 1
MC_EDGES_TSV = 2
MC_EDGES_SNAP = 3


class McError(RuntimeError):
    """A non-zero status returned by the C ABI."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {strerror(status)} (status {status})")


class Timing(C.Structure):
    _fields_ = [
        ("h2d_ms", C.c_double),
        ("orient_ms", C.c_double),
        ("count_ms", C.c_double),
        ("d2h_ms", C.c_double),
        ("total_ms", C.c_double),
        ("hub_ms", C.c_double),
        ("leaf_ms", C.c_double),
        ("launches", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TcStats(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("nnz", C.c_int64),
        ("dag_edges", C.c_int64),
        ("max_out_degree", C.c_int64),
        ("hub_tasks", C.c_int64),
        ("leaf_tasks", C.c_int64),
        ("partner_edges", C.c_int64),
        ("probe_work", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# name -> (restype, argtypes): every function include/mercury.h declares.
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_I64 = C.c_int64
_PI64 = C.POINTER(C.c_int64)
_PU64 = C.POINTER(C.c_uint64)
SIGNATURES = {
    "mc_strerror": (C.c_char_p, [C.c_int]),
    "mc_version": (C.c_char_p, []),
    "mc_graph_load": (C.c_int, [C.c_char_p, _PP]),
    "mc_graph_write": (C.c_int, [_P, C.c_char_p]),
    "mc_graph_from_csr": (C.c_int, [_P, _P, _I64, _I64, _PP]),
    "mc_graph_info": (C.c_int, [_P, _PI64, _PI64, _PI64]),
    "mc_graph_rowptr": (_P, [_P]),
    "mc_graph_col": (_P, [_P]),
    "mc_graph_validate": (C.c_int, [_P, C.c_int]),
    "mc_graph_load_vlabels": (C.c_int, [_P, C.c_char_p]),
    "mc_graph_vlabels": (C.c_int, [_P, _PP]),
    "mc_graph_free": (None, [_P]),
    "mc_gen_rmat": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, _PP]),
    "mc_gen_chung_lu": (C.c_int, [_I64, C.c_double, C.c_double, C.c_double, C.c_uint64, _PP]),
    "mc_edges_load": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _PP]),
    "mc_edges_from_arrays": (C.c_int, [_P, _P, _I64, _I64, _PP]),
    "mc_edges_info": (C.c_int, [_P, _PI64, _PI64]),
    "mc_edges_src": (_P, [_P]),
    "mc_edges_dst": (_P, [_P]),
    "mc_edges_free": (None, [_P]),
    "mc_gen_rmat_edges": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, _PP]),
    "mc_gen_chung_lu_edges": (C.c_int, [_I64, C.c_double, C.c_double, C.c_double, C.c_uint64, _PP]),
    "mc_csr_build": (C.c_int, [_P, _P, _I64, _I64, C.c_uint, _P, _PP, C.POINTER(Timing)]),
    "mc_dgraph_from_edges": (C.c_int, [_P, _P, _I64, _I64, C.c_uint, _P, _PP, C.POINTER(Timing)]),
    "mc_dgraph_create": (C.c_int, [_P, _P, _I64, _I64, _P, C.c_uint, _PP]),
    "mc_dgraph_create_device": (C.c_int, [_P, _P, _I64, _I64, _P, C.c_uint, _PP]),
    "mc_dgraph_stream": (C.c_int, [_P, _PP]),
    "mc_dgraph_info": (C.c_int, [_P, _PI64, _PI64, _PI64]),
    "mc_dgraph_export_csr": (C.c_int, [_P, _P, _P]),
    "mc_dgraph_columns_on_host": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "mc_dgraph_dag_on_host": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "mc_dgraph_free": (None, [_P]),
    "mc_tc_count": (C.c_int, [_P, _PU64, C.POINTER(Timing)]),
    "mc_tc_count_shard": (C.c_int, [_P, C.c_int, C.c_int, _PU64, C.POINTER(Timing)]),
    "mc_tc_stats": (C.c_int, [_P, C.POINTER(TcStats)]),
    "mc_dgraph_export_dag": (C.c_int, [_P, _P, _P]),
    "mc_tc_count_host": (C.c_int, [_P, _P, _I64, _I64, _PU64, C.POINTER(Timing)]),
    "mc_pattern_count": (C.c_int, [_P, C.c_int, _PU64, C.POINTER(Timing)]),
    "mc_pattern_count_shard": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _PU64, C.POINTER(Timing)]),
    "mc_pattern_count_budget": (C.c_int, [_P, C.c_int, C.c_double, _PU64,
                                          C.POINTER(C.c_double), C.POINTER(Timing)]),
    "mc_pattern_count_static": (C.c_int, [_P, _P, _I64, _I64, C.c_int, _PU64, _P]),
    "mc_batch_create": (C.c_int, [_P, _P, _I64, _I64, _P, C.c_int, _P, _P, _PP]),
    "mc_batch_autotune": (C.c_int, [_P, _P]),
    "mc_batch_count": (C.c_int, [_P, _PU64, C.POINTER(Timing)]),
    "mc_batch_free": (None, [_P]),
    "mc_dgraph_set_vlabels": (C.c_int, [_P, _P, C.c_int]),
    "mc_label_frequency": (C.c_int, [_P, _PU64]),
    "mc_label_reverse_index": (C.c_int, [_P, _P, _P]),
    "mc_label_nlf": (C.c_int, [_P, _I64, _I64, _P]),
    "mc_tc_count_by_label": (C.c_int, [_P, _PU64, C.POINTER(Timing)]),
    "mc_server_create": (C.c_int, [_I64, C.c_int, C.c_int, _PP]),
    "mc_server_submit": (C.c_int, [_P, _P, _P, _I64, _I64, C.c_int, C.c_uint64, _PU64]),
    "mc_server_wait": (C.c_int, [_P, C.c_uint64, C.c_int, _PU64, C.POINTER(C.c_double)]),
    "mc_server_stats": (C.c_int, [_P, _P]),
    "mc_server_free": (None, [_P]),
}


def lib() -> C.CDLL:
    """The loaded library (raises FileNotFoundError when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: run `python -c 'from mercury_b200.build import build; build()'` "
                "(or `make -C mercury_b200/csrc`) first; there is no CPU fallback")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def strerror(status: int) -> str:
    return lib().mc_strerror(status).decode()


def check(status: int, what: str) -> None:
    if status != MC_OK:
        raise McError(status, what)
