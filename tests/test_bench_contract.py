"""The measurement helpers of bench.py, on the CPU.

The roofline's algorithmic bytes follow the edge-iterator merge volume
pinned for this path: per DAG edge u->v, 12 B plus 4 B x (d+u + d+v), plus
8 B per row offset; the hub share counts only edges whose owner (the end with
the larger d+, ties to the larger id) has d+ above the leaf limit. These
tests restate that formula with plain loops on small DAGs from the oracle's
orientation and check the bench's vectorised form against it, and check the
other inputs of the bench line (peaks, the ncu record of the hub kernel,
the reference program's counts, the workload config), and that the CPU
reference arm maps nothing of the product library.
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


def _args(**kw):
    d = dict(scale=22, edge_factor=16, seed=1, host_columns=False)
    d.update(kw)
    return SimpleNamespace(**d)


def test_hub_counters_are_used_only_for_the_workload_they_were_captured_on(tmp_path, monkeypatch):
    prof = tmp_path / "hub.txt"
    prof.write_text("# ncu ...\ndram_bytes_per_launch = 2.5e10\nwarp_inst_per_launch = 8e9\n"
                    "ncu_duration_ms = 11.0\n")
    monkeypatch.setattr(bench, "HUB_DRAM_PROFILE", str(prof))
    rec = bench.hub_profile(_args())
    assert rec["dram_bytes_per_launch"] == 2.5e10 and rec["warp_inst_per_launch"] == 8e9
    for other in (_args(scale=24), _args(scale=18), _args(edge_factor=8), _args(seed=2),
                  _args(host_columns=True)):
        assert bench.hub_profile(other) is None


def test_hub_roofline_reports_measured_traffic_and_issue(tmp_path, monkeypatch):
    prof = tmp_path / "hub.txt"
    prof.write_text("dram_bytes_per_launch = 2.0e10\nwarp_inst_per_launch = 9.0e9\n"
                    "ncu_duration_ms = 10.5\n")
    monkeypatch.setattr(bench, "HUB_DRAM_PROFILE", str(prof))
    ab = {"b_hub": 1.7e11}
    roof = bench.hub_roofline(_args(), 10.0, ab, 6500.0, "measured", {"sm_mhz": 1965.0})
    assert roof["traffic"] == 2.0e10
    assert roof["achieved"] == pytest.approx(2.0e10 / 0.010 / 1e9)
    assert roof["frac"] == pytest.approx(roof["achieved"] / 6500.0) and roof["frac"] <= 1.2
    slots = 148 * 4 * 1965e6 * 0.010
    assert roof["issue"]["frac"] == pytest.approx(9.0e9 / slots)
    # The merge volume is kept as information only.
    assert roof["algorithmic_gbs"] == pytest.approx(1.7e11 / 0.010 / 1e9)
    # Without a record for the workload there is no traffic and no fraction.
    roof = bench.hub_roofline(_args(scale=20), 10.0, ab, 6500.0, "measured", {"sm_mhz": 1965.0})
    assert roof["traffic"] is None and roof["frac"] is None


def test_committed_hub_record_parses_when_present():
    if not os.path.exists(bench.HUB_DRAM_PROFILE):
        pytest.skip("no committed ncu record of the hub kernel yet")
    rec = bench.hub_profile(_args())
    assert rec is not None and rec["dram_bytes_per_launch"] > 0


def test_reference_count_record_matches_rmat_configs():
    assert bench.committed_reference_count(_args()) == 2109663139
    assert bench.committed_reference_count(_args(scale=16)) == 15715146
    assert bench.committed_reference_count(_args(scale=23)) is None
    assert bench.committed_reference_count(_args(seed=2)) is None


def test_reference_arm_maps_no_product_library():
    import subprocess
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '10', "
            "'--steps', '1', '--warmup', '1']; sys.path.insert(0, %r); import bench; "
            "bench.main(); print('MAPPED', open('/proc/self/maps').read().count('libmercury_b200'))"
            % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["config"]["m"] > 0
    assert lines[-1] == "MAPPED 0"


def test_workload_config_names_the_placement():
    a = SimpleNamespace(scale=22, edge_factor=16, seed=1, host_columns=False)
    cfg = bench.workload_config(a)
    assert "RMAT scale 22" in cfg["workload"] and "columns" not in cfg
    a.host_columns = True
    cfg = bench.workload_config(a)
    assert cfg["columns"] == "host" and "host memory" in cfg["workload"]


def loop_pattern_bytes(n, rp, col):
    nb = [set(col[rp[v]:rp[v + 1]].tolist()) for v in range(n)]
    d = [len(x) for x in nb]
    m2 = len(col)
    base = 8.0 * (n + 1) + 8.0 * m2
    edges = [(v0, int(v1)) for v0 in range(n) for v1 in col[rp[v0]:rp[v0 + 1]]]
    base += sum(4 * (d[v0] + d[v1]) for v0, v1 in edges)
    cost = lambda xs: sum(16 + 4 * d[x] for x in xs)  # noqa: E731
    out = {"P1": base + sum(cost(nb[v]) for v in range(n))}
    outer = sum(cost(nb[v0] - nb[v1]) for v0, v1 in edges)
    out["P2"] = out["P3"] = base + outer
    out["P4"] = base + sum(cost(nb[v0] - nb[v1]) for v0, v1 in edges if v1 < v0)
    inner = sum(cost(nb[v0] & nb[v1]) for v0, v1 in edges)
    for k in (5, 6, 7, 8):
        out[f"P{k}"] = base + inner
    return out


@pytest.mark.parametrize("n,p,seed", [(40, 0.3, 4), (120, 0.2, 5)])
def test_pattern_bytes_equal_the_loop_restatement(n, p, seed):
    rp, col = csr_from_edges(n, random_graph(n, p, seed))
    got = bench.pattern_bytes(np.asarray(rp), np.asarray(col))
    want = loop_pattern_bytes(n, np.asarray(rp), np.asarray(col))
    for k, v in want.items():
        assert got[k] == pytest.approx(v, rel=1e-12), k


def test_pattern_summary_records_an_error_instead_of_raising():
    """The P1-P8 summary that the triangle bench appends never fails the
    triangle-count line: without a device it returns the error."""
    s = bench.pattern_summary(steps=1, n=2000, mean=6.0, cap=50.0)
    if "error" not in s:  # a device is present
        assert set(s["per_pattern"]) == {f"P{k}" for k in range(1, 9)}


def test_clock_summary_takes_the_median_under_load_and_every_reason():
    rows = [(1965.0, 1965.0, []), (1950.0, 1965.0, ["sw_power_cap"]), (345.0, 1965.0, []),
            (1965.0, 1965.0, ["hw_slowdown"])]
    s = bench.clock_summary(rows)
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["samples"] == 4 and s["samples_under_load"] == 3
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert bench.clock_summary([], 1965.0)["reasons"] == ["unsampled"]


def test_nvml_sampler_reads_the_board_of_the_cuda_device(monkeypatch):
    """A fake NVML: the sampler finds the board by the CUDA device's UUID,
    decodes the throttle-reason bits and samples until the region ends."""
    import time
    import torch

    calls = {"uuid": None, "shutdown": 0}

    class FakeNvml:
        NVML_CLOCK_SM = 1

        def nvmlInit(self):
            pass

        def nvmlShutdown(self):
            calls["shutdown"] += 1

        def nvmlDeviceGetHandleByUUID(self, uuid):
            calls["uuid"] = uuid
            return "h"

        def nvmlDeviceGetMaxClockInfo(self, h, kind):
            return 1965

        def nvmlDeviceGetClockInfo(self, h, kind):
            return 1900

        def nvmlDeviceGetCurrentClocksEventReasons(self, h):
            return 0x4 | 0x40  # sw_power_cap, hw_thermal_slowdown

    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml())
    monkeypatch.setattr(torch.cuda, "get_device_properties",
                        lambda d: SimpleNamespace(uuid="1234-abcd"))
    s = bench.ClockSampler(0)
    assert isinstance(s, bench.NvmlClockSampler)
    with s:
        time.sleep(0.05)
    got = s.summary()
    assert calls["uuid"] == "GPU-1234-abcd" and calls["shutdown"] == 1
    assert got["sm_mhz"] == 1900.0 and got["sm_max_mhz"] == 1965.0
    assert got["samples"] >= 2
    assert got["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
