"""Generates the edge-list fixtures in tests/golden/edges/.

For each fixture this writes a seeded GraphChallenge-style TSV ("u<TAB>v<TAB>1",
1-based ids, with duplicate, reversed and self-loop lines). It then runs the
reference's own converter front end on it, datasets/tsv2mtx.py (TSV ->
networkx Graph -> Matrix Market), and keeps the .mtx it writes.

edges.json records, per fixture, the symmetric CSR that the networkx Graph
describes: ids shifted to 0-based, self-loops removed, rows sorted. It is
stored as sizes plus a SHA-256 of rowptr (int64) and col (int32). networkx
computes it here, independently of the oracle and of the library.

Needs the reference tree (for tsv2mtx.py), networkx and pandas, so it runs
in the development container, not on a GPU host.
Run from the repository root:  python tests/golden/make_edge_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "edges")
# The reference checkout: $MERCURY_REFERENCE_DIR, else "reference" beside the
# repository.
REFERENCE = os.environ.get("MERCURY_REFERENCE_DIR") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
TSV2MTX = os.path.join(REFERENCE, "datasets", "tsv2mtx.py")


def csr_digest(rowptr: np.ndarray, col: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, dtype="<i8").tobytes())
    h.update(np.ascontiguousarray(col, dtype="<i4").tobytes())
    return h.hexdigest()


def fixture_pairs(name: str, rng: np.random.Generator):
    """1-based (u, v) lines of each fixture."""
    if name == "dups":
        # Small dense-ish graph: repeated and reversed lines and self-loops.
        u = rng.integers(1, 41, 150)
        v = rng.integers(1, 41, 150)
        rep = rng.integers(0, 150, 40)
        u = np.concatenate([u, u[rep], v[rep[:20]], [5, 9, 9, 17, 40]])
        v = np.concatenate([v, v[rep], u[rep[:20]], [5, 9, 9, 17, 40]])
    elif name == "sparse_ids":
        # 60 distinct vertices scattered over ids up to 500: n comes from
        # the largest id, not from the number of distinct vertices.
        ids = np.sort(rng.choice(np.arange(1, 501), 60, replace=False))
        ids[-1] = 500
        u = ids[rng.integers(0, 60, 200)]
        v = ids[rng.integers(0, 60, 200)]
    elif name == "hub":
        # A hub adjacent to 1,300 vertices (its row spans several 512-key
        # warp spans of the device build) plus random edges among the rest.
        u = np.concatenate([np.full(1300, 7), rng.integers(1, 1500, 900)])
        v = np.concatenate([rng.permutation(np.arange(1, 1501))[:1300],
                            rng.integers(1, 1500, 900)])
    else:
        raise KeyError(name)
    return u.astype(np.int64), v.astype(np.int64)


def networkx_csr(mtx_path: str, n: int):
    """CSR (0-based) of the graph networkx wrote, read back with networkx."""
    import networkx as nx

    g = nx.Graph()
    with open(mtx_path) as f:
        lines = [ln for ln in f if not ln.startswith("%")]
    for ln in lines[1:]:
        a, b = ln.split()[:2]
        g.add_edge(int(a), int(b))
    rowptr = np.zeros(n + 1, dtype=np.int64)
    cols = []
    for v in range(n):
        nb = sorted(x - 1 for x in g.neighbors(v + 1) if x != v + 1) if g.has_node(v + 1) else []
        cols.extend(nb)
        rowptr[v + 1] = rowptr[v] + len(nb)
    return rowptr, np.asarray(cols, dtype=np.int32)


def main():
    if not os.path.exists(TSV2MTX):
        sys.exit(f"{TSV2MTX} not found: this script needs the reference tree")
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(20240611)
    meta = {}
    for name in ("dups", "sparse_ids", "hub"):
        u, v = fixture_pairs(name, rng)
        tsv = os.path.join(OUT, name + ".tsv")
        with open(tsv, "w") as f:
            for a, b in zip(u, v):
                f.write(f"{a}\t{b}\t1\n")
        with tempfile.TemporaryDirectory() as tmp:
            shutil.copy(tsv, os.path.join(tmp, name + ".tsv"))
            subprocess.run([sys.executable, TSV2MTX, os.path.join(tmp, name)], check=True,
                           stdout=subprocess.DEVNULL)
            shutil.copy(os.path.join(tmp, name + ".mtx"), os.path.join(OUT, name + ".mtx"))
        n = int(max(u.max(), v.max()))  # 1-based ids: n = largest id
        rowptr, col = networkx_csr(os.path.join(OUT, name + ".mtx"), n)
        meta[name] = {"lines": int(len(u)), "n": n, "nnz": int(len(col)),
                      "max_degree": int(np.diff(rowptr).max()),
                      "self_loop_lines": int((u == v).sum()),
                      "csr_sha256": csr_digest(rowptr, col)}
        print(name, meta[name])
    with open(os.path.join(OUT, "edges.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
