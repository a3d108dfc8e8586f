"""Oracle counts of the hub test graph used by tests/test_zz_no_alloc.py.

The graph: vertex 0 adjacent to every other vertex 1..hub_degree, plus
3 * hub_degree seeded random pairs among 1..hub_degree (duplicates and
self-loops dropped).  One vertex of degree 20,000 makes the allocation-free
entry point run fewer blocks than the GPU holds.  P2 and P3 are left out:
their per-edge loops are quadratic in |N(0) - N(v)|, hours on this graph.

  python tests/golden/make_hub_golden.py   # writes tests/golden/hub_counts.json
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

HUB_DEGREE = 20000
PATTERNS = (1, 4, 5, 6, 7, 8)


def hub_graph(hub_degree=HUB_DEGREE, extra=3, seed=5):
    from oracle import oracle as orc
    rng = np.random.default_rng(seed)
    n = hub_degree + 1
    m = extra * hub_degree
    src = np.concatenate([np.zeros(hub_degree, dtype=np.int64), rng.integers(1, n, m)])
    dst = np.concatenate([np.arange(1, n, dtype=np.int64), rng.integers(1, n, m)])
    return orc.csr_from_edges(src, dst, n)


def main():
    from oracle import oracle as orc
    rp, col = hub_graph()
    out = {"hub_degree": HUB_DEGREE, "n": len(rp) - 1, "nnz": int(len(col)),
           "counts": {f"P{k}": orc.pattern(rp, col, k) for k in PATTERNS}}
    with open(os.path.join(HERE, "hub_counts.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
