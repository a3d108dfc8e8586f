"""mercury_b200 -- B200-native (sm_100a) counting path of GPM-lib/Mercury.

Triangle counting and the P1..P8 pattern counts on one GPU, behind the C ABI
of include/mercury.h (shared library in mercury_b200/lib/).  This package is
the Python host side of that ABI; the drop-in programs ``tc_challenge`` and
``sm`` are built into mercury_b200/bin/.
"""
from ._ffi import McError, Timing, lib  # noqa: F401
from .graph import DeviceGraph, Graph, TCSolver, tc_count_host  # noqa: F401
from .batch import Batch, union_csr  # noqa: F401
from .server import Server  # noqa: F401
from .edges import EdgeList, csr_build, dgraph_from_edges  # noqa: F401

__version__ = "0.1.0"
