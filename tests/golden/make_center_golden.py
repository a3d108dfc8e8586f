"""Expected P1..P8 counts (the oracle's) of the center-class test graph.

The graph (tests/test_patterns_gpu.py:center_class_graph) has one center
vertex in each degree class of the bitmap kernels (degrees 20 .. 900) and one
hub above 1024 (the warp-per-edge kernel), all attached to a sparse pool.
The oracle's P3 costs O(sum d^3) here (about a minute on 8 cores), too slow
to recompute in every test run, so the counts are stored in
center_counts.json.

Run from the repository root:  python tests/golden/make_center_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as orc  # noqa: E402
from test_patterns_gpu import center_class_graph  # noqa: E402


def main():
    rp, col = center_class_graph()
    out = {f"P{k}": int(orc.pattern(rp, col, k)) for k in range(1, 9)}
    out["n"], out["nnz"] = len(rp) - 1, len(col)
    print(out)
    with open(os.path.join(HERE, "center_counts.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
