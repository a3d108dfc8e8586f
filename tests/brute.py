"""Brute-force counts for tiny graphs, independent of the oracle's code.

Enumerates every 3-, 4- and 5-vertex subset, classifies its induced subgraph
up to isomorphism and combines the counts into the quantities the reference's
pattern formulas compute (each derived by following the set algebra of
subgraph_matching/pattern_kernels.cuh over all 2m directed edges):

  TC = triangles                      P1 = claws (K1,3)
  P2 = forks (chairs)                 P3 = 4*K1,4 + 3*claws
  P4 = induced 4-paths                P5 = 2*bulls
  P6 = 2*paws + 2*(diamond with a pendant on a chord vertex)
  P7 = 2*K1,1,3                       P8 = 3*tailed K4
"""
from __future__ import annotations

import itertools

import numpy as np


def _edges_to_mask(k, edges):
    m = 0
    for a, b in edges:
        a, b = min(a, b), max(a, b)
        m |= 1 << _pair_index(k, a, b)
    return m


_PAIR = {}


def _pair_index(k, a, b):
    key = (k, a, b)
    if key not in _PAIR:
        idx = 0
        for i in range(k):
            for j in range(i + 1, k):
                _PAIR[(k, i, j)] = idx
                idx += 1
    return _PAIR[key]


def _canon(k, adj_bits):
    """Smallest pair-mask over all vertex permutations."""
    best = None
    pairs = [(i, j) for i in range(k) for j in range(i + 1, k)]
    for perm in itertools.permutations(range(k)):
        m = 0
        for i, j in pairs:
            if adj_bits[i][j]:
                a, b = perm[i], perm[j]
                if a > b:
                    a, b = b, a
                m |= 1 << _pair_index(k, a, b)
        if best is None or m < best:
            best = m
    return best


def _canon_edges(k, edges):
    adj = [[False] * k for _ in range(k)]
    for a, b in edges:
        adj[a][b] = adj[b][a] = True
    return _canon(k, adj)


TARGETS = {
    "triangle": (3, [(0, 1), (1, 2), (0, 2)]),
    "claw": (4, [(0, 1), (0, 2), (0, 3)]),
    "p4": (4, [(0, 1), (1, 2), (2, 3)]),
    "paw": (4, [(0, 1), (1, 2), (0, 2), (0, 3)]),
    "k14": (5, [(0, 1), (0, 2), (0, 3), (0, 4)]),
    "fork": (5, [(0, 1), (0, 2), (0, 3), (3, 4)]),
    "bull": (5, [(0, 1), (1, 2), (0, 2), (0, 3), (1, 4)]),
    # diamond {0,1,2,3} with chord 0-1, pendant 4 on chord vertex 1
    "diamond_pendant": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (1, 4)]),
    "k113": (5, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4)]),
    "tailed_k4": (5, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (0, 4)]),
}
_TARGET_CANON = {name: (k, _canon_edges(k, e)) for name, (k, e) in TARGETS.items()}


def induced_counts(rowptr, col) -> dict:
    n = len(rowptr) - 1
    adj = [set(col[rowptr[v]:rowptr[v + 1]].tolist()) for v in range(n)]
    counts = {name: 0 for name in TARGETS}
    by_k = {}
    for name, (k, c) in _TARGET_CANON.items():
        by_k.setdefault(k, {})[c] = name
    for k in (3, 4, 5):
        if n < k:
            continue
        wanted = by_k[k]
        for sub in itertools.combinations(range(n), k):
            bits = [[(sub[j] in adj[sub[i]]) for j in range(k)] for i in range(k)]
            ne = sum(bits[i][j] for i in range(k) for j in range(i + 1, k))
            if ne < 3:
                continue
            c = _canon(k, bits)
            if c in wanted:
                counts[wanted[c]] += 1
    return counts


def expected_from_counts(c: dict) -> dict:
    return {
        "TC": c["triangle"],
        "P1": c["claw"],
        "P2": c["fork"],
        "P3": 4 * c["k14"] + 3 * c["claw"],
        "P4": c["p4"],
        "P5": 2 * c["bull"],
        "P6": 2 * c["paw"] + 2 * c["diamond_pendant"],
        "P7": 2 * c["k113"],
        "P8": 3 * c["tailed_k4"],
    }


def triangles(rowptr, col) -> int:
    n = len(rowptr) - 1
    adj = [set(col[rowptr[v]:rowptr[v + 1]].tolist()) for v in range(n)]
    t = 0
    for u in range(n):
        for v in adj[u]:
            if v > u:
                t += sum(1 for w in adj[v] if w > v and w in adj[u])
    return t


def random_graph(n, p, seed):
    rng = np.random.default_rng(seed)
    edges = [(i, j) for i in range(n) for j in range(i + 1, n) if rng.random() < p]
    return edges
