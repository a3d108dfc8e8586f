"""The hub triangle kernel's work, counted on the CPU (tests/hub_work.cpp).

The kernel's scheduling choices are claims about work: pairing long partner
lists by length class needs fewer 128-entry pair batches than row order;
giving each warp one contiguous range of the short stream takes fewer list
steps than interleaved windows; the dense-partner AND replaces list probes
with at most dense_factor words per entry.  These tests check those claims
on RMAT graphs, and that the restated decomposition covers exactly the
partner work an independent numpy count gives.  Run as a script, it prints
the figures for RMAT scale 22 (edge factor 16, seed 1) that the design notes
quote:  python tests/test_hub_work.py [scale]
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

FIELDS = ("hub_tasks", "short_lists", "short_entries", "long_lists", "long_entries",
          "dense_partners", "dense_probes", "dense_words", "steps_between_windows",
          "steps_inside_windows", "steps_ranges", "pair_batches_row", "pair_batches_classes",
          "pair_batches_sorted", "dense_quad_slots_claims", "dense_quad_slots_own")
# The kernel's defaults: 32 KB of bitmap less the probe's zero quad, 32,768
# core ranks, 2 words per entry.
BITMAP_BITS, CORE_RANKS, DENSE_FACTOR = 32768 * 8 - 128, 32768, 2

_lib = None


def lib():
    global _lib
    if _lib is None:
        out = os.path.join(HERE, "_build", "libhub_work.so")
        src = os.path.join(HERE, "hub_work.cpp")
        if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
            os.makedirs(os.path.dirname(out), exist_ok=True)
            subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", src,
                            "-o", out], check=True)
        _lib = C.CDLL(out)
    return _lib


def hub_work(rowptr, col, bitmap_bits=BITMAP_BITS, core_ranks=CORE_RANKS,
             dense_factor=DENSE_FACTOR) -> dict:
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    ci = np.ascontiguousarray(col, dtype=np.int32)
    out = np.zeros(len(FIELDS))
    lib().hub_work(C.c_int64(len(rp) - 1), C.c_void_p(rp.ctypes.data), C.c_void_p(ci.ctypes.data),
                   C.c_int(bitmap_bits), C.c_int(core_ranks), C.c_int(dense_factor),
                   C.c_void_p(out.ctypes.data))
    return {k: int(v) for k, v in zip(FIELDS, out)}


def partner_work_numpy(rowptr, col):
    """Sum of d+(y) over the partners y of owners with d+ > 64, and their
    number of row chunks of 512 (hub tasks), counted independently."""
    rp, ci = np.asarray(rowptr, np.int64), np.asarray(col, np.int64)
    n = len(rp) - 1
    deg = np.diff(rp)
    src = np.repeat(np.arange(n), deg)
    keep = (deg[ci] > deg[src]) | ((deg[ci] == deg[src]) & (ci > src))
    dp = np.bincount(src[keep], minlength=n)
    px, py = dp[src], dp[ci]
    partner = (py >= 1) & ((px > py) | ((px == py) & (src > ci))) & (px > 64)
    tasks = int(((deg + 511) // 512)[dp > 64].sum())
    return int(py[partner].sum()), tasks


@pytest.mark.parametrize("scale,seed", [(12, 1), (14, 3)])
def test_decomposition_covers_the_partner_work(scale, seed):
    from mercury_b200 import Graph
    g = Graph.rmat(scale, 16, seed=seed)
    w = hub_work(g.rowptr, g.col)
    work, tasks = partner_work_numpy(g.rowptr, g.col)
    assert w["hub_tasks"] == tasks
    assert w["long_entries"] + w["short_entries"] + w["dense_probes"] == work
    assert w["dense_words"] <= DENSE_FACTOR * w["dense_probes"]
    assert 4 * w["dense_quad_slots_own"] >= w["dense_words"]
    assert w["dense_quad_slots_claims"] >= w["dense_quad_slots_own"]
    # Without core bitmaps every long partner is streamed.
    w0 = hub_work(g.rowptr, g.col, core_ranks=0)
    assert w0["dense_partners"] == 0
    assert w0["long_entries"] == w["long_entries"] + w["dense_probes"]


def test_scheduling_choices_reduce_the_work():
    from mercury_b200 import Graph
    g = Graph.rmat(15, 16, seed=1)
    w = hub_work(g.rowptr, g.col)
    assert w["short_lists"] > 0
    assert w["steps_ranges"] < w["steps_between_windows"] + w["steps_inside_windows"]
    # At this size every long partner ranks inside the core: without core
    # bitmaps they are all streamed in pairs.
    w0 = hub_work(g.rowptr, g.col, core_ranks=0)
    assert w0["long_lists"] > 0
    assert w0["pair_batches_sorted"] <= w0["pair_batches_classes"] < w0["pair_batches_row"]


if __name__ == "__main__":
    from mercury_b200 import Graph
    scale = int(sys.argv[1]) if len(sys.argv) > 1 else 22
    g = Graph.rmat(scale, 16, seed=1)
    for k, v in hub_work(g.rowptr, g.col).items():
        print(f"{k:24s} {v:>16,d}")
