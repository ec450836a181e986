"""The CPU oracle against the reference's own outputs (no GPU).

The golden counts in tests/golden/counts.json were printed by the reference's
`patternmatchcpu -a 0` built from its sources (tests/golden/make_golden.py).
"""
import numpy as np
import pytest

import oracle_py as O
from conftest import golden_graph_path



def test_k6_closed_forms(golden):
    # counts of subgraphs of K6: C(6,3), 3*C(6,4), 6*C(6,4), C(6,4), house, C(6,5)
    c = golden["k6"]["counts"]
    assert (c["0"], c["1"], c["2"], c["3"], c["4"], c["7"]) == (20, 45, 90, 15, 360, 6)


def test_k20_reference_counts_and_closed_forms(golden):
    # K20 is the reference's own cross-check graph (its Q5 count must agree
    # between the CPU algorithms, TestPatternMatchCPU.cpp:97-147); the clique
    # counts are binomials, the 4-cycle 3*C(n,4), the diamond 6*C(n,4), the
    # house 5!/2 * C(n,5)
    from math import comb
    c = golden["k20"]["counts"]
    assert c["0"] == comb(20, 3) and c["3"] == comb(20, 4) and c["7"] == comb(20, 5) and c["11"] == comb(20, 6)
    assert c["1"] == 3 * comb(20, 4) and c["2"] == 6 * comb(20, 4) and c["4"] == 60 * comb(20, 5)
    rp, cl = O.read_bin(golden_graph_path("k20"))
    assert O.count(rp, cl, 5) == c["5"] == 13953600


def test_oracle_matches_reference_counts(golden):
    # every golden count (about 90 s on 8 host threads for the largest ones)
    checked = 0
    for name, d in golden.items():
        rp, cl = O.read_bin(golden_graph_path(name))
        for q, want in d["counts"].items():
            assert O.count(rp, cl, int(q)) == want, (name, q)
            checked += 1
    assert checked >= 120


def test_oracle_enumeration_consistent(golden):
    rp, cl = O.read_bin(golden_graph_path("er_n64_d12"))
    for q in (0, 1, 2, 3, 4, 7):
        inst = O.enumerate_sorted(rp, cl, q)
        assert len(inst) == golden["er_n64_d12"]["counts"][str(q)]
        # every instance is injective and edge-preserving
        assert all(len(set(r)) == len(r) for r in inst.tolist())
        assert len(np.unique(inst, axis=0)) == len(inst)


def test_oracle_root_ranges_partition_the_count(golden):
    rp, cl = O.read_bin(golden_graph_path("rmat_s10_ef8"))
    n = len(rp) - 1
    total = O.count(rp, cl, 3)
    cut = [0, 17, 200, n // 2, n]
    parts = sum(O.count(rp, cl, 3, root_begin=a, root_end=b) for a, b in zip(cut, cut[1:]))
    assert parts == total == golden["rmat_s10_ef8"]["counts"]["3"]
