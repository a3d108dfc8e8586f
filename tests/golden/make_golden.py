"""Generates the golden fixtures in tests/golden/.

Writes each fixture graph in the reference's on-disk CSR layout
(graphs/<name>/graph.meta.txt, graph.vertex.bin int64[n+1],
graph.edge.bin int32[nnz]; graph.cc:18-35) with numpy, independently of the
library's writer, and golden.json with the expected counts:
  * tiny graphs: brute-force induced-subgraph counts (tests/brute.py), which
    must agree with the oracle before anything is written;
  * larger graphs: the oracle (oracle/oracle.cpp, oracle/patterns_oracle.cpp).
Counts from the reference's own programs run on a GPU go to
reference_counts.json (tests/golden/run_reference.py).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from brute import expected_from_counts, induced_counts, random_graph  # noqa: E402
from conftest import csr_from_edges  # noqa: E402
from oracle import oracle as orc  # noqa: E402

PATTERNS = [f"P{k}" for k in range(1, 9)]


def write_triple(prefix, rowptr, col):
    n = len(rowptr) - 1
    md = int(np.diff(rowptr).max()) if n else 0
    os.makedirs(os.path.dirname(prefix), exist_ok=True)
    with open(prefix + ".meta.txt", "w") as f:
        f.write(f"{n} {len(col)} 4 8 1 2 {md} 0 0 0\n")
    np.asarray(rowptr, dtype=np.int64).tofile(prefix + ".vertex.bin")
    np.asarray(col, dtype=np.int32).tofile(prefix + ".edge.bin")


def rmat_edges(scale, ef, seed, a=0.57, b=0.19, c=0.19):
    rng = np.random.default_rng(seed)
    m = ef << scale
    src = np.zeros(m, dtype=np.int64)
    dst = np.zeros(m, dtype=np.int64)
    for _ in range(scale):
        r = rng.random(m)
        sb = (r >= a + b).astype(np.int64)
        db = (((r >= a) & (r < a + b)) | (r >= a + b + c)).astype(np.int64)
        src = (src << 1) | sb
        dst = (dst << 1) | db
    return list(zip(src.tolist(), dst.tolist()))


def chung_lu_edges(n, mean, cap, gamma, seed):
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (gamma - 1.0))
    w = np.minimum(w * mean * n / w.sum(), cap)
    p = w / w.sum()
    m = int(n * mean / 2)
    s = rng.choice(n, size=m, p=p)
    d = rng.choice(n, size=m, p=p)
    return list(zip(s.tolist(), d.tolist()))


def fixtures():
    out = {}
    out["k5"] = csr_from_edges(5, [(i, j) for i in range(5) for j in range(i + 1, 5)])
    out["star9"] = csr_from_edges(9, [(0, i) for i in range(1, 9)])
    out["path6"] = csr_from_edges(6, [(i, i + 1) for i in range(5)])
    pet = [(i, (i + 1) % 5) for i in range(5)] + [(i, i + 5) for i in range(5)] + \
          [(5 + i, 5 + (i + 2) % 5) for i in range(5)]
    out["petersen"] = csr_from_edges(10, pet)
    out["rand13"] = csr_from_edges(13, random_graph(13, 0.45, 11))
    # isolated vertices inside and at the end (trailing empty rows)
    out["isolated"] = csr_from_edges(16, [(1, 3), (3, 5), (1, 5), (5, 7), (7, 9), (9, 11),
                                          (5, 9), (1, 7), (3, 7)])
    out["rmat8"] = csr_from_edges(256, rmat_edges(8, 8, 7))
    out["rmat10"] = csr_from_edges(1024, rmat_edges(10, 16, 1))
    out["cl3000"] = csr_from_edges(3000, chung_lu_edges(3000, 8.0, 300.0, 2.1, 5))
    out["dense400"] = csr_from_edges(400, random_graph(400, 0.55, 3))
    return out


TINY = {"k5", "star9", "path6", "petersen", "rand13", "isolated"}
TC_ONLY = {"dense400"}


def main():
    golden = {}
    for name, (rp, col) in fixtures().items():
        write_triple(os.path.join(HERE, "graphs", name, "graph"), rp, col)
        rec = {"n": len(rp) - 1, "nnz": int(len(col)), "TC": orc.tc(rp, col),
               "division": orc.division(rp, col)}
        if name not in TC_ONLY:
            for k in range(1, 9):
                rec[f"P{k}"] = orc.pattern(rp, col, k)
        if name in TINY:
            exp = expected_from_counts(induced_counts(rp, col))
            got = {k: rec[k] for k in exp}
            assert exp == got, (name, exp, got)
            rec["source"] = "brute-force induced counts == oracle"
        else:
            rec["source"] = "oracle"
        golden[name] = rec
        print(name, {k: v for k, v in rec.items() if k != "division"}, flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
