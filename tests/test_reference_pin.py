"""The oracle pinned to the reference's own programs.

tests/golden/reference_counts.json holds the counts printed by the
reference's tc_challenge and pattern kernels (built from the reference
sources for sm_100a by oracle/ref.mk and run on a B200 by
tests/golden/run_reference.py).  The oracle must reproduce every one.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as orc

with open(os.path.join(GOLDEN, "reference_counts.json")) as f:
    REF = json.load(f)
with open(os.path.join(GOLDEN, "golden.json")) as f:
    GOLD = json.load(f)

CHEAP = {"k5", "star9", "path6", "petersen", "rand13", "isolated", "rmat8"}


def load(name):
    prefix = os.path.join(GOLDEN, "graphs", name, "graph")
    return (np.fromfile(prefix + ".vertex.bin", dtype=np.int64),
            np.fromfile(prefix + ".edge.bin", dtype=np.int32))


@pytest.mark.parametrize("name", sorted(REF["fixtures"]))
def test_golden_counts_equal_reference_program_output(name):
    for key, val in REF["fixtures"][name].items():
        assert GOLD[name][key] == val, (name, key)


@pytest.mark.parametrize("name", sorted(REF["fixtures"]))
def test_oracle_reproduces_reference_program(name):
    rp, col = load(name)
    ref = REF["fixtures"][name]
    assert orc.tc(rp, col) == ref["TC"]
    if name in CHEAP:
        for k in range(1, 9):
            assert orc.pattern(rp, col, k) == ref[f"P{k}"], (name, k)


def test_oracle_reproduces_reference_on_rmat16():
    from mercury_b200 import Graph
    g = Graph.rmat(16, 16, seed=1)
    rec = REF["rmat_tc"]["rmat16"]
    assert g.n == rec["n"] and g.nnz // 2 == rec["m"]
    assert orc.tc(g.rowptr, g.col) == rec["triangles"]
