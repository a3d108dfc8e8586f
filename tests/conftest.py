import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size case (minutes)")


def _built() -> bool:
    return os.path.exists(os.path.join(ROOT, "mercury_b200", "lib", "libmercury_b200.so"))


@pytest.fixture(scope="session", autouse=True)
def _build_once():
    """Build the library and the oracle once per session if they are missing."""
    if not _built():
        from mercury_b200.build import build
        build()
    from oracle import oracle as orc
    orc.lib()


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def csr_from_edges(n, edges):
    """Symmetric, sorted, deduplicated CSR from undirected edge pairs."""
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    cols = []
    for v in range(n):
        nb = sorted(adj[v])
        rowptr[v + 1] = rowptr[v] + len(nb)
        cols.extend(nb)
    return rowptr, np.array(cols, dtype=np.int32)


def relabel(rowptr, col, perm):
    """The same graph with vertex v renamed perm[v] (rows re-sorted)."""
    n = len(rowptr) - 1
    deg = np.diff(rowptr)
    src = np.repeat(np.arange(n), deg)
    ns, nd = perm[src], perm[col]
    order = np.lexsort((nd, ns))
    ns, nd = ns[order], nd[order]
    rp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rp, ns + 1, 1)
    return np.cumsum(rp), nd.astype(np.int32)
