"""The restated per-edge terms of the warp-per-edge pattern kernels, on the CPU.

The kernels' fast forms (mercury_b200/csrc/patterns.cu) do not evaluate the
reference's loops (subgraph_matching/pattern_kernels.cuh) term by term. They
rewrite each count through the symmetry of the graph, for example
#{c in C : c not in N(b)} = |C| - |N(b) & C|, or read it off bit rows over
A. This file restates those forms literally in Python and checks that, summed
over all directed edges and combined as the reference combines them
(sm_multigpu.cu:206-232), they give the oracle's P4-P8 counts, 32-bit
products included. The GPU tests check the kernels against the same oracle.
"""
import numpy as np
import pytest

from brute import random_graph
from conftest import csr_from_edges
from oracle import oracle as orc

MASK64 = (1 << 64) - 1


def wrap_mul(a, b):
    """The reference's int x int product, wrapped to 32 bits and sign-extended."""
    p = (a * b) & 0xFFFFFFFF
    return p - (1 << 32) if p >= 1 << 31 else p


def neighbourhoods(rp, col):
    n = len(rp) - 1
    return [set(int(x) for x in col[rp[v]:rp[v + 1]]) for v in range(n)]


def directed_edges(rp, col):
    for v0 in range(len(rp) - 1):
        for e in range(rp[v0], rp[v0 + 1]):
            yield v0, int(col[e])


def p4(N, edges):
    c1 = 0
    for v0, v1 in edges:
        if v1 >= v0:
            continue
        A, B = N[v0] - N[v1], N[v1] - N[v0]
        outer, inner = (A, B) if len(A) < len(B) else (B, A)
        for v2 in outer:  # ni - |N(v2) & inner|
            c1 += len(inner) - len(N[v2] & inner)
    return c1 & MASK64


def p5(N, edges):
    c1 = c2 = 0
    for v0, v1 in edges:
        A, B, C = N[v0] & N[v1], N[v0] - N[v1], N[v1] - N[v0]
        if A:
            for b in B:  # f = nA - |N(b) & A|, t = nC - |N(b) & C|
                f = len(A) - len(N[b] & A)
                if f:
                    c1 += wrap_mul(len(C) - len(N[b] & C), f)
        for v2 in A:  # D = C & N(v2), E = B - N(v2)
            D, E = C & N[v2], B - N[v2]
            for c in D:
                c2 += len(E) - len(N[c] & E)
    return (c1 - c2) & MASK64


def p6(N, edges):
    c1 = 0
    for v0, v1 in edges:
        A, B = N[v0] & N[v1], N[v1] - N[v0]
        for v2 in A:
            D, E = A - N[v2], B - N[v2]
            outer, inner = (D, E) if len(D) < len(E) else (E, D)
            for v3 in outer:
                c1 += len(inner) - len(N[v3] & inner)
    return c1 & MASK64


def rows_within(N, A):
    """M[i] = {k : A[k] in N(A[i])} as bit masks over the ascending A."""
    return [sum(1 << k for k, y in enumerate(A) if y in N[x]) for x in A]


def popc(x):
    return bin(x).count("1")


def p7(N, edges):
    c1 = c2 = 0
    for v0, v1 in edges:
        A = sorted(N[v0] & N[v1])
        n = len(A)
        assert n <= 32
        M = rows_within(N, A)
        valid = (1 << n) - 1
        for i in range(n):
            below = (1 << i) - 1
            above = valid & ~below & ~(1 << i)
            freq = popc(~M[i] & above)
            c = popc(~M[i] & below)
            c1 += wrap_mul(c, freq)
            d = ~M[i] & below
            for t in range(n):
                if M[i] >> t & 1:
                    c2 += popc(d & (valid & ~((2 << t) - 1)) & ~M[t])
    return (c1 - c2) & MASK64


def p8(N, edges):
    c1 = c2 = 0
    for v0, v1 in edges:
        A = sorted(N[v0] & N[v1])
        B = sorted(N[v1] - N[v0])
        assert len(A) <= 32
        M = rows_within(N, A)
        for j, x in enumerate(A):  # freq = nB - |N(a) & B|, c = |N(a) & A below a|
            hb = len(N[x] & set(B))
            ca = popc(M[j] & ((1 << j) - 1))
            c1 += wrap_mul(ca, len(B) - hb)
        above = [~((2 << i) - 1) & ((1 << len(A)) - 1) for i in range(len(A))]
        for b in B:  # mask_C over A; sum over i in C of popc(M[i] above i & ~mask_C)
            mc = sum(1 << k for k, y in enumerate(A) if b in N[y])
            for i in range(len(A)):
                if mc >> i & 1:
                    c2 += popc(M[i] & above[i] & ~mc)
    return (c1 - c2) & MASK64


FORMS = {4: p4, 5: p5, 6: p6, 7: p7, 8: p8}


@pytest.mark.parametrize("n,p,seed", [(24, 0.3, 1), (40, 0.25, 2), (40, 0.45, 3), (60, 0.15, 4)])
@pytest.mark.parametrize("k", sorted(FORMS))
def test_restated_forms_equal_the_oracle(n, p, seed, k):
    rp, col = csr_from_edges(n, random_graph(n, p, seed))
    rp, col = np.asarray(rp), np.asarray(col)
    N = neighbourhoods(rp, col)
    assert FORMS[k](N, list(directed_edges(rp, col))) == orc.pattern(rp, col, k)


def clique_form(rp, col, k):
    """P7 or P8 as the clique route of mercury_b200/csrc/cliques.cu computes
    them, restated literally: triangles listed once on the degree-ordered DAG
    (u -> v -> w), a_e = |N(x) & N(y)| per edge, k_tau = |N(u) & N(v) & N(w)|
    per triangle, and the K5s (u, v, w, x, y) with x, y in N+(u) & N+(v) &
    N+(w) and y in N+(x); every term added modulo 2^64."""
    N = neighbourhoods(rp, col)
    n = len(N)
    deg = [len(s) for s in N]
    out = [{w for w in N[u] if deg[w] > deg[u] or (deg[w] == deg[u] and w > u)}
           for u in range(n)]
    a = {}
    for u in range(n):
        for v in out[u]:
            a[frozenset((u, v))] = len(N[u] & N[v])
    acc = 0
    if k == 7:
        acc += sum(2 * (t * (t - 1) * (t - 2) // 6) for t in a.values())
    for u in range(n):
        for v in out[u]:
            for w in out[u] & out[v]:
                kt = len(N[u] & N[v] & N[w])
                sum_a = a[frozenset((u, v))] + a[frozenset((u, w))] + a[frozenset((v, w))]
                S = out[u] & out[v] & out[w]
                k5 = sum(len(S & out[x]) for x in S)
                if k == 7:
                    acc += 6 * (kt * (kt - 1) // 2) - kt * (sum_a - 6) - 20 * k5
                else:
                    acc += kt * (deg[u] + deg[v] + deg[w]) - 3 * kt * sum_a + 9 * kt * kt - 60 * k5
    return acc & MASK64


@pytest.mark.parametrize("n,p,seed", [(14, 0.5, 31), (22, 0.4, 32), (30, 0.35, 33),
                                      (40, 0.25, 34)])
@pytest.mark.parametrize("k", [7, 8])
def test_clique_route_forms_equal_the_oracle(n, p, seed, k):
    """The clique route's per-edge and per-triangle terms give the oracle's
    P7 and P8 on random graphs (the GPU tests check the kernels too)."""
    rp, col = csr_from_edges(n, random_graph(n, p, seed))
    assert clique_form(rp, col, k) == orc.pattern(rp, col, k)
