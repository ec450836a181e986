"""GPU parity of the enumeration engine through the C-ABI (libsme.so).

Counts are compared bit-exactly with the reference's own CPU program (golden
counts) and with the C oracle; instance lists are compared sorted.
"""
import numpy as np
import pytest

import oracle_py as O
import subgraphmatchgpu_b200 as sme
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu

ALGOS = (sme.GPU_GPSM, sme.GPU_GPSM_REUSE, sme.GPU_LIGHT)
GPU_LIMIT = 3_000_000_000


@pytest.fixture(scope="module")
def graphs(golden):
    return {name: sme.Graph.load(golden_graph_path(name)) for name in golden}


@pytest.mark.parametrize("algo", ALGOS)
def test_counts_match_reference_on_golden_graphs(graphs, golden, algo):
    for name, d in golden.items():
        g = graphs[name]
        for q, want in d["counts"].items():
            if want > GPU_LIMIT:
                continue
            got = g.count(int(q), algo, reuse_autogen=-1)
            assert got == want, (name, q, algo, got, want)


@pytest.mark.parametrize("gran", [1, 2, 3])
def test_intersection_granularities(graphs, golden, gran):
    # 1: warp per path generic, 2: flattened over 32 paths per warp (specialised),
    # 3: specialised warp per path at six blocks per SM (0, auto, runs in
    # every other test)
    for name in ("rmat_s12_ef8", "ba_n600_m4", "k12"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            for algo in ALGOS:
                assert graphs[name].count(int(q), algo, warp_granularity=gran) == want, (name, q, algo, gran)
    rp, cl = O.read_bin(golden_graph_path("er_n64_d12"))
    for q in (0, 3, 4):
        got = O.sort_rows(graphs["er_n64_d12"].enumerate(q, sme.GPU_LIGHT, warp_granularity=gran))
        assert np.array_equal(got, O.enumerate_sorted(rp, cl, q))


@pytest.mark.parametrize("root_map", ["0", "1"])
def test_root_list_bitmap_and_warp_kernel_agree(graphs, golden, root_map, monkeypatch):
    # two-list steps on the root's list run k_compute_rootmap by default
    # (the root's list as a shared-memory bitmap); SME_ROOT_MAP=0 sends them
    # to the warp-per-path kernel.  Both give the reference's counts, and
    # the same sorted instances (write steps).
    monkeypatch.setenv("SME_ROOT_MAP", root_map)
    for name in ("rmat_s12_ef8", "ba_n600_m4", "er_n600_d8", "k20"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            for algo in ALGOS:
                got = graphs[name].count(int(q), algo)
                assert got == want, (name, q, algo, root_map, got, want)
    for name in ("er_n64_d12", "ba_n600_m4"):
        rp, cl = O.read_bin(golden_graph_path(name))
        for q in (0, 1, 2, 3, 7):
            want = O.enumerate_sorted(rp, cl, q)
            for algo in ALGOS:
                got = O.sort_rows(graphs[name].enumerate(q, algo))
                assert got.shape == want.shape and np.array_equal(got, want), (name, q, algo, root_map)


@pytest.mark.parametrize("threshold", ["32", "256"])
def test_long_pivot_paths_on_a_cta_each(graphs, golden, threshold, monkeypatch):
    # granularity 4: two-list steps hand paths whose clipped pivot holds at
    # least SME_HEAVY_PIVOT elements to a CTA each (the other list staged in
    # shared memory by a bulk copy when it is not a hub); a low threshold
    # sends many paths there on the small graphs
    monkeypatch.setenv("SME_HEAVY_PIVOT", threshold)
    for name in ("rmat_s12_ef8", "ba_n600_m4", "rmat_s10_ef8", "k20"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            for algo in ALGOS:
                got = graphs[name].count(int(q), algo, warp_granularity=4)
                assert got == want, (name, q, algo, threshold, got, want)
                got = graphs[name].count(int(q), algo, warp_granularity=4, list_only=1)
                assert got == want, (name, q, algo, threshold, "list_only", got, want)
    for name in ("er_n64_d12", "ba_n600_m4"):
        rp, cl = O.read_bin(golden_graph_path(name))
        for q in (0, 3, 4, 2):
            got = O.sort_rows(graphs[name].enumerate(q, sme.GPU_LIGHT, warp_granularity=4))
            assert np.array_equal(got, O.enumerate_sorted(rp, cl, q)), (name, q)


@pytest.mark.parametrize("level", [0, 1, 2, 3])
def test_light_compress_levels(graphs, golden, level):
    for name in ("rmat_s10_ef8", "ba_n600_m4", "k12"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            assert graphs[name].count(int(q), sme.GPU_LIGHT, compress_level=level) == want, (name, q, level)


@pytest.mark.parametrize("level", [0, 3])
def test_light_without_set_reuse(graphs, golden, level):
    # every candidate set from adjacency lists, as the reference computes them
    for name in ("rmat_s10_ef8", "ba_n600_m4", "k12", "er_n64_d12"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            got = graphs[name].count(int(q), sme.GPU_LIGHT, compress_level=level, no_set_reuse=1)
            assert got == want, (name, q, level)


def test_reuse_autogen_plans(graphs, golden):
    for name in ("rmat_s10_ef8", "er_n64_d12"):
        for q, want in golden[name]["counts"].items():
            if want > GPU_LIMIT:
                continue
            assert graphs[name].count(int(q), sme.GPU_GPSM_REUSE, reuse_autogen=1) == want, (name, q)


@pytest.mark.parametrize("algo", ALGOS)
def test_sorted_instances_identical_to_oracle(graphs, algo):
    for name in ("er_n64_d12", "k6", "ba_n600_m4"):
        rp, cl = O.read_bin(golden_graph_path(name))
        for q in (0, 1, 2, 3, 4, 7, 6, 9):
            want = O.enumerate_sorted(rp, cl, q)
            got = O.sort_rows(graphs[name].enumerate(q, algo))
            assert got.shape == want.shape and np.array_equal(got, want), (name, q, algo)


def test_ordering_disabled_counts_automorphic_images(graphs):
    # -r 0: every automorphic image is counted (Query::DisableOrdering)
    rp, cl = O.read_bin(golden_graph_path("er_n64_d12"))
    for q in (0, 1, 3, 4):
        want = O.count(rp, cl, q, ordering=False)
        for algo in ALGOS:
            assert graphs["er_n64_d12"].count(q, algo, enable_ordering=0) == want


def test_root_ranges_sum_to_total(graphs, golden):
    g = graphs["rmat_s12_ef8"]
    n = g.n
    for q in (0, 3, 1):
        cuts = [0, 5, 100, n // 3, n]
        parts = sum(g.count(q, sme.GPU_LIGHT, root_begin=a, root_end=b) for a, b in zip(cuts, cuts[1:]))
        assert parts == golden["rmat_s12_ef8"]["counts"][str(q)]


@pytest.mark.parametrize("q", [5, 9, 10, 13])
def test_reuse_plan_locates_sibling_caches(graphs, golden, q):
    # the hard-coded reuse plans of Q5, Q9, Q10 and Q13 reuse, at a later
    # level, the level-2 intersection N(M0) ∩ N(M[x]) a sibling path cached;
    # the engine finds it by rank in N(M0) and falls back to the adjacency
    # lists when the sibling is in another batch (a small budget forces many)
    name = "rmat_s10_ef8"
    want = golden[name]["counts"][str(q)]
    g = graphs[name]
    assert "sibling=(2" in sme.plan_describe(q, 6).split("algo=5")[1].split("program")[0]
    assert g.count(q, sme.GPU_GPSM_REUSE) == want
    hits = sme.last_stats().reuse_hits
    assert hits > 0
    # six-vertex patterns need a larger arena for one path's level buffers
    budget = (4 << 20) if q in (9, 10) else (8 << 20)
    assert g.count(q, sme.GPU_GPSM_REUSE, mem_limit_bytes=budget) == want
    assert sme.last_stats().batches > 1
    for name2 in ("ba_n600_m4", "er_n64_d12", "k12"):
        w = golden[name2]["counts"].get(str(q))
        if w is not None and w <= GPU_LIMIT:
            assert graphs[name2].count(q, sme.GPU_GPSM_REUSE) == w, name2


def test_small_memory_budget_forces_many_batches(graphs, golden):
    g = graphs["rmat_s12_ef8"]
    for algo in ALGOS:
        for q in (3, 1, 4):
            got = g.count(q, algo, mem_limit_bytes=24 << 20)
            assert got == golden["rmat_s12_ef8"]["counts"][str(q)], (algo, q)
            assert sme.last_stats().batches > 3


def test_auto_budget_after_a_small_budget_call(graphs, golden):
    # a call with the auto budget must not inherit the previous call's arena
    g = graphs["rmat_s12_ef8"]
    want = golden["rmat_s12_ef8"]["counts"]["3"]
    assert g.count(3, sme.GPU_LIGHT, mem_limit_bytes=8 << 20) == want
    small_batches = sme.last_stats().batches
    assert g.count(3, sme.GPU_LIGHT) == want
    assert sme.last_stats().batches < small_batches


def test_failed_upload_releases_the_arena():
    # a graph that is not resident is uploaded into the call's arena; when it
    # does not fit, the call fails with OOM and the arena is whole again
    big = sme.Graph.rmat(16, 16, seed=3)
    with pytest.raises(sme.SmeError) as e:
        big.count(3, mem_limit_bytes=4 << 20)
    assert e.value.status == 3
    small = sme.Graph.clique(12)
    for _ in range(3):
        assert small.count(3, mem_limit_bytes=4 << 20) == 495


@pytest.mark.parametrize("algo", [sme.GPU_GPSM_REUSE, sme.GPU_LIGHT])
def test_partitioned_counts(graphs, golden, algo):
    # -m 0: the total over the graph, and per partition the instances inside it
    name = "rmat_s12_ef8"
    g = graphs[name]
    n = g.n
    part = (np.arange(n) * 7 % 4).astype(np.uint32)
    for q in (0, 3, 4):
        total, intra = g.count_partitioned(q, part, 4, algo=algo)
        assert total == golden[name]["counts"][str(q)]
        for p in range(4):
            assert intra[p] == O.count(*g.partition(part, p).csr(), q), (q, p)
        assert intra.sum() <= total


def test_edge_cases():
    # empty-ish, single edge, star, path, triangle
    def csr(n, edges):
        adj = [[] for _ in range(n)]
        for u, v in edges:
            adj[u].append(v)
            adj[v].append(u)
        rp = np.zeros(n + 1, np.uint64)
        for u in range(n):
            rp[u + 1] = rp[u] + len(adj[u])
        cl = np.array([v for u in range(n) for v in sorted(adj[u])], np.uint32)
        return rp, cl

    cases = {
        "single_edge": (2, [(0, 1)]),
        "star": (9, [(0, i) for i in range(1, 9)]),
        "path": (7, [(i, i + 1) for i in range(6)]),
        "triangle": (3, [(0, 1), (1, 2), (0, 2)]),
        "two_k4": (8, [(a, b) for a in range(4) for b in range(a + 1, 4)] +
                   [(a, b) for a in range(4, 8) for b in range(a + 1, 8)]),
    }
    for name, (n, e) in cases.items():
        rp, cl = csr(n, e)
        g = sme.Graph.from_csr(rp, cl)
        for q in (0, 1, 2, 3, 4, 7):
            want = O.count(rp, cl, q)
            for algo in ALGOS:
                assert g.count(q, algo) == want, (name, q, algo)
    g = sme.Graph.from_csr(np.zeros(1, np.uint64), np.zeros(0, np.uint32))
    assert g.count(0) == 0


def test_graph_with_self_loops_keeps_injectivity_checks():
    # the != checks against list owners are dropped only for loop-free graphs;
    # with self loops a vertex is in its own list and the checks must stay
    rp, cl = O.read_bin(golden_graph_path("er_n64_d12"))
    n = len(rp) - 1
    adj = [set(cl[rp[u]:rp[u + 1]].tolist()) for u in range(n)]
    for u in range(0, n, 3):
        adj[u].add(u)
    lrp = np.zeros(n + 1, np.uint64)
    for u in range(n):
        lrp[u + 1] = lrp[u] + len(adj[u])
    lcl = np.array([v for u in range(n) for v in sorted(adj[u])], np.uint32)
    g = sme.Graph.from_csr(lrp, lcl)
    for q in (0, 1, 2, 3, 4, 7):
        want = O.count(lrp, lcl, q)
        for algo in ALGOS:
            assert g.count(q, algo) == want, (q, algo)


def test_resident_graph_and_stats():
    g = sme.Graph.rmat(14, 8, seed=1)
    rp, cl = g.csr()
    want = O.count(rp, cl, 0)
    assert g.count(0) == want
    s0 = sme.last_stats()
    assert s0.h2d_bytes > 0
    g.to_device(0)
    assert g.count(0) == want
    s = sme.last_stats()
    assert s.h2d_bytes == 0 and s.kernel_launches > 0 and s.algorithmic_bytes > 0
    for algo in ALGOS:
        assert g.count(0, algo) == want


def test_plans_agree_at_scale():
    g = sme.Graph.rmat(16, 16, seed=3)
    g.to_device(0)
    for q in (0, 2, 3, 7):
        c = [g.count(q, a) for a in ALGOS]
        assert c[0] == c[1] == c[2], (q, c)


def test_invalid_options_fail_cleanly():
    g = sme.Graph.clique(5)
    with pytest.raises(sme.SmeError) as e:
        g.count(14)
    assert e.value.status == 6
    with pytest.raises(sme.SmeError):
        g.count(0, algo=3)
    with pytest.raises(sme.SmeError):
        g.count(0, mode=0)
    with pytest.raises(sme.SmeError) as e:
        g.count(1, sme.GPU_GPSM_REUSE, reuse_autogen=0)
    assert e.value.status == 6
    # the context stays usable
    assert g.count(0) == 10
