"""mc_pattern_count_static: the pattern count for callers that may not
allocate device memory (a host application whose own pool owns the GPU's
memory, or a latency-bound caller that cannot pay for cudaMalloc/cudaFree).
It must give the same uint64 counts as mc_pattern_count, and the golden
(oracle) counts, while taking all its scratch from the library's fixed
device array -- on small graphs, where the grid is bounded by occupancy, and
on a graph with a vertex of degree 20,000, where the array holds room for only
8 blocks of frontier lists (8 MiB ints / (8 warps x 6 lists x 20,000)), fewer
than the GPU holds.

This file is collected after every other test file, so a run that stops at
the first failure has already run the rest.
"""
import ctypes as C
import os

import numpy as np
import pytest

import json
import sys

from conftest import GOLDEN
from mercury_b200 import DeviceGraph, Graph
from mercury_b200 import _ffi

sys.path.insert(0, GOLDEN)
from make_hub_golden import PATTERNS as HUB_PATTERNS, hub_graph  # noqa: E402

with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)
with open(os.path.join(GOLDEN, "hub_counts.json")) as f:
    HUB = json.load(f)

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch
    rp = torch.from_numpy(np.array(g.rowptr)).cuda()
    col = torch.from_numpy(np.array(g.col)).cuda()
    torch.cuda.synchronize()
    return rp, col


def _static_count(rp, col, n, nnz, k, stream=None):
    out = C.c_uint64()
    rc = _ffi.lib().mc_pattern_count_static(rp.data_ptr(), col.data_ptr(), n, nnz, k,
                                            C.byref(out), stream)
    _ffi.check(rc, f"static pattern P{k}")
    return out.value


@pytest.mark.parametrize("name", ["rmat8", "cl3000", "rand13", "isolated"])
def test_static_entry_matches_allocating_entry_twice(name):
    import torch
    g = Graph(os.path.join(GOLDEN, "graphs", name, "graph"))
    with DeviceGraph(g) as d:
        want = [d.pattern_count(k) for k in range(1, 9)]
    rp, col = _device_csr(g)
    first = [_static_count(rp, col, g.n, g.nnz, k) for k in range(1, 9)]
    free_before, _ = torch.cuda.mem_get_info()
    second = [_static_count(rp, col, g.n, g.nnz, k) for k in range(1, 9)]
    free_after, _ = torch.cuda.mem_get_info()
    assert first == want
    assert second == want  # the shared scratch keeps no state between calls
    assert free_after == free_before  # nothing was allocated by the second round
    for k in range(1, 9):
        if f"P{k}" in GOLD[name]:
            assert first[k - 1] == GOLD[name][f"P{k}"], (name, k)


def test_static_entry_with_fewer_blocks_than_the_gpu_holds_on_a_stream():
    """One vertex of degree 20,000: the array fits 8 blocks of frontier lists.
    The first round runs on a torch stream (non-NULL cudaStream_t), the
    second on the default stream; both equal the oracle's counts and the
    allocating entry point's."""
    import torch
    rp_h, col_h = hub_graph()
    assert HUB["n"] == len(rp_h) - 1 and HUB["nnz"] == len(col_h)
    g = Graph.from_csr(rp_h, col_h)
    rp, col = _device_csr(g)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        first = {k: _static_count(rp, col, g.n, g.nnz, k, C.c_void_p(s.cuda_stream))
                 for k in HUB_PATTERNS}
    second = {k: _static_count(rp, col, g.n, g.nnz, k) for k in HUB_PATTERNS}
    with DeviceGraph(g) as d:
        want = {k: d.pattern_count(k) for k in HUB_PATTERNS}
    for k in HUB_PATTERNS:
        assert first[k] == HUB["counts"][f"P{k}"], k
        assert second[k] == first[k] == want[k], k


def test_static_entry_rejects_bad_input_and_oversized_degree():
    import torch
    # pattern id out of range
    g = Graph(os.path.join(GOLDEN, "graphs", "k5", "graph"))
    rp, col = _device_csr(g)
    out = C.c_uint64()
    rc = _ffi.lib().mc_pattern_count_static(rp.data_ptr(), col.data_ptr(), g.n, g.nnz, 9,
                                            C.byref(out), None)
    assert rc == _ffi.MC_ERR_ARG
    # a vertex id outside [0, n) is caught before any pattern kernel runs
    bad = torch.tensor([1, 7], dtype=torch.int32, device="cuda")
    brp = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = _ffi.lib().mc_pattern_count_static(brp.data_ptr(), bad.data_ptr(), 2, 2, 1,
                                            C.byref(out), None)
    assert rc == _ffi.MC_ERR_FORMAT
    # a star whose hub degree (200000) leaves no room for a block of frontier lists
    n = 200001
    rp_h = np.zeros(n + 1, dtype=np.int64)
    rp_h[1] = n - 1
    rp_h[2:] = n - 1 + np.arange(1, n)
    col_h = np.concatenate([np.arange(1, n), np.zeros(n - 1)]).astype(np.int32)
    srp = torch.from_numpy(rp_h).cuda()
    scol = torch.from_numpy(col_h).cuda()
    torch.cuda.synchronize()
    rc = _ffi.lib().mc_pattern_count_static(srp.data_ptr(), scol.data_ptr(), n, len(col_h), 4,
                                            C.byref(out), None)
    assert rc == _ffi.MC_ERR_UNSUPPORTED
