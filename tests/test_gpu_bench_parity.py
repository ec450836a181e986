"""Counts on the bench's own configurations, every plan and mode, against the
CPU oracle on the same root tasks.

The R-MAT scale-20 graph is the bench's (numpy generator, the engine's
preprocessing); R-MAT scale 16 and 18 use the same generator.  Whole-graph
counts at these scales take the oracle minutes to hours, so each case counts
the same root task on both sides: a strided task (every k-th root from an
offset, the shape of an IntraPartScheduler task) or an explicit block of the
bench's own root permutation.  Offsets are chosen away from the R-MAT hub ids
(ids with few set bits), whose single-root DFS keeps the oracle busy for
minutes.
"""
import functools
import os
import sys

import numpy as np
import pytest

import oracle_py as O
import subgraphmatchgpu_b200 as sme

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

PLANS = (sme.GPU_GPSM, sme.GPU_GPSM_REUSE, sme.GPU_LIGHT)


@functools.lru_cache(maxsize=None)
def engine_graph(scale, seed):
    args = bench.parse(["--scale", str(scale), "--seed", str(seed)])
    g = bench.engine_graph(args)
    g.to_device(0)
    return g, args


@pytest.fixture(scope="module")
def s20():
    g, args = engine_graph(20, 20)
    rp, cl = g.csr()
    return g, args, rp, cl


def run_all(g, q, want, **task):
    """Every plan in memory, and LIGHT in external mode (the only plan the
    external mode runs), on the same task.  A task's roots are the vertices
    of the plan's first pattern vertex: u0 in every plan but the LIGHT house
    (Q4), which starts at u1 (its search sequence is 1 2 3 0 4), so for Q4
    only the plans rooted at u0 count the oracle's task."""
    for algo in (PLANS if q != 4 else (sme.GPU_GPSM, sme.GPU_GPSM_REUSE)):
        got = g.count(q, algo, **task)
        assert got == want, (q, algo, task.get("root_begin"), got, want)
    if q == 4:
        return
    got = g.count(q, sme.GPU_LIGHT, mode=sme.EXTERNAL_GPU, **task)
    assert got == want, (q, "external", got, want)
    # long-pivot paths on a CTA each (granularity 4)
    got = g.count(q, sme.GPU_LIGHT, warp_granularity=4, **task)
    assert got == want, (q, "granularity 4", got, want)


@pytest.mark.parametrize("q", [3, 1, 2])
@pytest.mark.parametrize("offset", [717, 939])
def test_s20_strided_tasks_match_oracle(s20, q, offset):
    g, _, rp, cl = s20
    stride = 1024
    want = O.count_strided(rp, cl, q, stride, offset)
    run_all(g, q, want, root_begin=offset, root_stride=stride)


@pytest.mark.parametrize("q", [3, 1, 2])
def test_s20_bench_root_blocks_match_oracle(s20, q):
    # the first block of the bench's own step list for each query
    g, args, rp, cl = s20
    steps = bench.make_steps(rp, args, 3)
    roots = next(r for qq, r in steps if qq == q)
    if q == 3:
        roots = roots[:4096]
    want = O.count_roots(rp, cl, q, roots)
    run_all(g, q, want, roots=roots)


@pytest.mark.parametrize("scale,stride,offsets,queries", [
    (16, 64, (37, 59), (0, 1, 2, 3, 7)),
    (16, 4096, (2059,), (4,)),  # the house: 16 roots keep the oracle to seconds
    (18, 256, (173, 221), (0, 1, 2, 3)),
])
def test_s16_s18_strided_tasks_match_oracle(scale, stride, offsets, queries):
    g, _ = engine_graph(scale, scale)
    rp, cl = g.csr()
    for q in queries:
        for off in offsets:
            want = O.count_strided(rp, cl, q, stride, off)
            run_all(g, q, want, root_begin=off, root_stride=stride)


def test_explicit_root_task_counts_each_listed_root():
    # a root listed twice counts twice; order does not matter; ids >= n fail
    g = sme.Graph.rmat(12, 8, seed=13)
    rp, cl = g.csr()
    roots = np.array([5, 17, 5, 100, 3], np.uint32)
    want = sum(O.count(rp, cl, 3, root_begin=int(r), root_end=int(r) + 1) for r in roots)
    for algo in PLANS:
        assert g.count(3, algo, roots=roots) == want
        assert g.count(3, algo, roots=roots[::-1]) == want
    with pytest.raises(sme.SmeError) as e:
        g.count(3, roots=np.array([g.n], np.uint32))
    assert e.value.status == 1


def test_count_steps_grouped_by_hub(monkeypatch):
    # SME_GROUP_BY_HUB=1: a count step takes its paths grouped by the hub
    # whose bitmap it probes (a counting sort of the frontier); the count is
    # the same in any order
    g, _ = engine_graph(16, 16)
    want = {q: g.count(q, sme.GPU_LIGHT) for q in (3, 2, 1)}
    monkeypatch.setenv("SME_GROUP_BY_HUB", "1")
    for q, w in want.items():
        assert g.count(q, sme.GPU_LIGHT) == w, q
        assert g.count(q, sme.GPU_GPSM) == w, q
