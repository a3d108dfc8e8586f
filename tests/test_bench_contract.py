"""The measurement helpers of bench.py, on the CPU.

The roofline's algorithmic bytes follow the edge-iterator merge volume
pinned for this path: per DAG edge u->v, 12 B plus 4 B x (d+u + d+v), plus
8 B per row offset; the hub share counts only edges whose owner (the end with
the larger d+, ties to the larger id) has d+ above the leaf limit. These
tests restate that formula with plain loops on small DAGs from the oracle's
orientation and check the bench's vectorised form against it, and check the
other inputs of the bench line (peaks, committed traffic, workload config).
"""
import json
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from brute import random_graph
from conftest import ROOT, csr_from_edges
from oracle import oracle as orc

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def loop_bytes(n, drp, dcol, leaf_max):
    dplus = [int(drp[v + 1] - drp[v]) for v in range(n)]
    b_tc = 8.0 * (n + 1)
    b_hub, hub_edges, owners = 0.0, 0, set()
    for u in range(n):
        for e in range(drp[u], drp[u + 1]):
            v = int(dcol[e])
            du, dv = dplus[u], dplus[v]
            b_tc += 12 + 4 * (du + dv)
            if du >= 1 and dv >= 1:
                owner = u if (du > dv or (du == dv and u > v)) else v
                if dplus[owner] > leaf_max:
                    b_hub += 12 + 4 * (du + dv)
                    hub_edges += 1
                    owners.add(owner)
    return b_tc, b_hub + 8.0 * len(owners), hub_edges


@pytest.mark.parametrize("n,p,seed", [(60, 0.3, 1), (200, 0.5, 2), (400, 0.45, 3)])
def test_algorithmic_bytes_equal_the_loop_restatement(n, p, seed):
    rp, col = csr_from_edges(n, random_graph(n, p, seed))
    drp, dcol = orc.orient(np.asarray(rp), np.asarray(col))
    got = bench.algorithmic_bytes(n, drp, dcol)
    b_tc, b_hub, hub_edges = loop_bytes(n, drp, dcol, bench.LEAF_MAX_OUT)
    assert got["b_tc"] == b_tc
    assert got["b_hub"] == b_hub
    assert got["hub_edges"] == hub_edges
    assert got["b_min"] <= got["b_tc"]
    if n >= 200:
        assert hub_edges > 0  # dense enough for owners above the leaf limit


def test_peaks_come_from_the_measured_file_when_present():
    peak, kind = bench.load_peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            assert peak == float(json.load(f)["hbm_gbs"])
        assert kind == "measured"
    else:
        assert (peak, kind) == (6650.0, "fallback")


def test_traffic_is_read_from_the_committed_hub_profile():
    t = bench.traffic_from_profile()
    assert t is not None and t > 0
    with open(os.path.join(ROOT, "profiles", "tc_hub_kernel_rmat22.txt")) as f:
        line = [ln for ln in f if ln.startswith("dram_bytes_per_launch")][0]
    assert t == float(line.split("=")[1].split()[0])


def test_workload_config_names_the_placement():
    a = SimpleNamespace(scale=22, edge_factor=16, seed=1, host_columns=False)
    cfg = bench.workload_config(a)
    assert "RMAT scale 22" in cfg["workload"] and "columns" not in cfg
    a.host_columns = True
    cfg = bench.workload_config(a)
    assert cfg["columns"] == "host" and "host memory" in cfg["workload"]
