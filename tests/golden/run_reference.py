"""Runs the reference's own programs (built from its sources into oracle/_ref/
by oracle/ref.mk) on a GPU and records their counts and runtimes.

  python tests/golden/run_reference.py [--out reference_run.json]
                                       [--scales 16,20,22] [--repeats 3]

* Fixture counts: oracle/_ref/tc_challenge and oracle/_ref/sm_patterns
  (P1..P8) on every graph in tests/golden/graphs; their
  "total_num_triangles = N" lines are collected.  The committed result is
  tests/golden/reference_counts.json (the oracle is pinned to it by
  tests/test_reference_pin.py).
* Timing: RMAT graphs of the listed scales (edge factor 16, seed 1, the
  library's generator) are written in the reference's file layout and run
  through the reference's tc_challenge and this repository's tc_challenge;
  the "Runtime  = X sec" lines are collected.

The reference's triangle program runs only on graphs whose DAG out-degrees
are all <= 128.  Above that, tc_challenge.cu:93-101 sends vertices to
hashIndex_for_large_degree (gpu_kernels/tc_challenge.cuh:4-192), which reads
as racy: after the bin scan (offsets 1, 2, ..., 512: ten rounds, so the
result sits in the first half of shared_bucket), one loop packs each bin's
offset from shared_bucket[0..1019) and the next loop, with no barrier between
them, copies the table over shared_bucket from index 0.  A warp that is
still packing can read a vertex id as an offset, and the copy then writes
outside the 16 KB buffer.  The kernel faulted on a B200 (error 700 at
tc_challenge.cu:103) on RMAT scales 22 and 24.  Every vertex with out-degree
above 128 reaches that kernel, so no such graph is run; their counts come
from tests/golden/reference_counts.json, where earlier runs of the same
program recorded them (and the oracle reproduces each one).  The pattern
shim (oracle/ref_sm_shim.cu) does not use that kernel and still runs.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF_TC = os.path.join(ROOT, "oracle", "_ref", "tc_challenge")
REF_SM = os.path.join(ROOT, "oracle", "_ref", "sm_patterns")
OUR_TC = os.path.join(ROOT, "mercury_b200", "bin", "tc_challenge")
COUNT = re.compile(r"total_num_triangles = (\d+)")
RUNTIME = re.compile(r"^Runtime  = ([0-9.eE+-]+) sec", re.M)
SM_RUNTIME = re.compile(r"^Total runtime  = ([0-9.eE+-]+) sec", re.M)


def run(cmd, timeout):
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return None, "timeout"
    if r.returncode != 0:
        return None, f"exit {r.returncode}: {r.stderr.strip()[-300:]}"
    return r.stdout, None


# Largest DAG out-degree for which tc_challenge.cu routes no vertex to the
# hash kernel (the DEG_THD split of graph.cc:237-312).
REF_TC_MAX_OUT = 128


def reference_tc_limits_ok(rowptr, col):
    """(run?, why): the reference triangle program runs only when no vertex
    has a DAG out-degree above 128, so that its hash kernel, whose staging
    loops race (gpu_kernels/tc_challenge.cuh:76-94), has no tasks."""
    from oracle import oracle as orc
    drp, _ = orc.orient(rowptr, col)
    top = int(np.diff(drp).max(initial=0))
    if top > REF_TC_MAX_OUT:
        return False, (f"max d+ {top} > {REF_TC_MAX_OUT}: the graph reaches the reference's "
                       f"hash kernel, whose staging loops race")
    return True, f"max d+ {top}"


def recorded_tc(key):
    """Count the reference program printed earlier for this graph, if any."""
    with open(os.path.join(HERE, "reference_counts.json")) as f:
        rec = json.load(f)
    if key in rec.get("fixtures", {}):
        return rec["fixtures"][key].get("TC")
    r = rec.get("rmat_tc", {}).get(key)
    return None if r is None else r["triangles"]


def fixture_counts(timeout):
    out = {}
    gdir = os.path.join(HERE, "graphs")
    golden = json.load(open(os.path.join(HERE, "golden.json")))
    for name in sorted(os.listdir(gdir)):
        prefix = os.path.join(gdir, name, "graph")
        rp = np.fromfile(prefix + ".vertex.bin", dtype=np.int64)
        col = np.fromfile(prefix + ".edge.bin", dtype=np.int32)
        rec = {}
        ok, why = reference_tc_limits_ok(rp, col)
        rec["tc_limits"] = why
        if ok:
            s, err = run([REF_TC, prefix], timeout)
            rec["TC"] = int(COUNT.search(s).group(1)) if s else err
        elif recorded_tc(name) is not None:
            rec["TC"] = recorded_tc(name)
            rec["tc_source"] = "recorded earlier (reference_counts.json)"
        for k in range(1, 9):
            if f"P{k}" not in golden[name]:
                continue
            s, err = run([REF_SM, prefix, f"P{k}"], timeout)
            rec[f"P{k}"] = int(COUNT.search(s).group(1)) if s else err
        out[name] = rec
        print(name, rec, flush=True)
    return out


def timing(scales, repeats, timeout):
    from mercury_b200 import Graph
    res = {}
    with tempfile.TemporaryDirectory() as tmp:
        for sc in scales:
            g = Graph.rmat(sc, 16, seed=1)
            prefix = os.path.join(tmp, f"rmat{sc}", "graph")
            os.makedirs(os.path.dirname(prefix))
            g.write(prefix)
            rec = {"n": g.n, "m": g.nnz // 2}
            ok, why = reference_tc_limits_ok(np.asarray(g.rowptr), np.asarray(g.col))
            rec["ref_limits"] = why
            for label, exe, allowed in (("reference", REF_TC, ok), ("ours", OUR_TC, True)):
                if not allowed:
                    rec[label] = "skipped: " + why
                    if recorded_tc(f"rmat{sc}") is not None:
                        rec["reference_recorded_count"] = recorded_tc(f"rmat{sc}")
                    continue
                runs = []
                for _ in range(repeats):
                    s, err = run([exe, prefix], timeout)
                    if s is None:
                        runs.append(err)
                        break
                    runs.append({"runtime_s": float(RUNTIME.search(s).group(1)),
                                 "count": int(COUNT.search(s).group(1))})
                rec[label] = runs
            res[f"rmat{sc}"] = rec
            print(f"rmat{sc}", rec, flush=True)
    return res


OUR_SM = os.path.join(ROOT, "mercury_b200", "bin", "sm")
SM_RUNTIME_ANY = re.compile(r"Total runtime  = ([0-9.eE+-]+) sec")


def pattern_timing(n, mean, cap, repeats, timeout):
    """The reference's pattern kernels and this build's `sm` on one seeded
    Chung-Lu graph (the generator bench.py --mode patterns uses)."""
    from mercury_b200 import Graph
    g = Graph.chung_lu(n, 2.1, mean, cap, seed=1)
    res = {"n": g.n, "m": g.nnz // 2, "max_degree": g.max_degree}
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "cl", "graph")
        os.makedirs(os.path.dirname(prefix))
        g.write(prefix)
        for k in range(1, 9):
            rec = {}
            for label, exe in (("reference", REF_SM), ("ours", OUR_SM)):
                best = None
                for _ in range(repeats):
                    s, err = run([exe, prefix, f"P{k}"], timeout)
                    if s is None:
                        best = err
                        break
                    t = float(SM_RUNTIME_ANY.search(s).group(1))
                    c = int(COUNT.search(s).group(1))
                    if best is None or t < best["runtime_s"]:
                        best = {"runtime_s": t, "count": c}
                rec[label] = best
            res[f"P{k}"] = rec
            print(f"P{k}", rec, flush=True)
    return res


def tc_chung_lu_timing(n, repeats, timeout):
    from mercury_b200 import Graph
    g = Graph.chung_lu(n, 2.1, 20.0, 50000.0, seed=1)
    rec = {"n": g.n, "m": g.nnz // 2, "max_degree": g.max_degree}
    ok, why = reference_tc_limits_ok(np.asarray(g.rowptr), np.asarray(g.col))
    rec["ref_limits"] = why
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "cl", "graph")
        os.makedirs(os.path.dirname(prefix))
        g.write(prefix)
        for label, exe, allowed in (("reference", REF_TC, ok), ("ours", OUR_TC, True)):
            if not allowed:
                rec[label] = "skipped: " + why
                continue
            runs = []
            for _ in range(repeats):
                s, err = run([exe, prefix], timeout)
                if s is None:
                    runs.append(err)
                    break
                runs.append({"runtime_s": float(RUNTIME.search(s).group(1)),
                             "count": int(COUNT.search(s).group(1))})
            rec[label] = runs
    print("chung-lu", rec, flush=True)
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--patterns", default="", help="n,mean,cap of a Chung-Lu graph to time P1..P8")
    ap.add_argument("--tc-chung-lu", type=int, default=0, help="vertices of a Chung-Lu TC timing")
    ap.add_argument("--out", default="reference_run.json")
    ap.add_argument("--scales", default="16,20,22")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--timeout", type=float, default=120.0)
    ap.add_argument("--skip-fixtures", action="store_true")
    a = ap.parse_args()
    result = {}
    if not a.skip_fixtures:
        result["fixtures"] = fixture_counts(a.timeout)
    scales = [int(s) for s in a.scales.split(",") if s]
    if scales:
        result["timing"] = timing(scales, a.repeats, a.timeout)
    if a.patterns:
        pn, pm, pc = a.patterns.split(",")
        result["patterns"] = pattern_timing(int(pn), float(pm), float(pc), a.repeats, a.timeout)
    if a.tc_chung_lu:
        result["tc_chung_lu"] = tc_chung_lu_timing(a.tc_chung_lu, a.repeats, a.timeout)
    if os.path.dirname(a.out):
        os.makedirs(os.path.dirname(a.out), exist_ok=True)
    with open(a.out, "w") as f:
        json.dump(result, f, indent=1)


if __name__ == "__main__":
    main()
