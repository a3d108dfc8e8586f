"""The C-ABI library loads and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

from conftest import ROOT
from mercury_b200 import _ffi

DECL = re.compile(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(mc_[a-z_0-9]+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(DECL.findall(src))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["mc_graph_load", "mc_dgraph_create", "mc_tc_count", "mc_tc_count_host",
                 "mc_strerror"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(_ffi.SIGNATURES)


def test_strerror_and_version_need_no_gpu():
    assert _ffi.strerror(_ffi.MC_ERR_FORMAT) == "input breaks the CSR contract"
    assert b"sm_100a" in _ffi.lib().mc_version()
