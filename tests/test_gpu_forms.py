"""External (chunked) mode, batched form and served form on the GPU, each
checked bit-exactly against the reference counts / the C oracle."""
import random

import numpy as np
import pytest

import oracle_py as O
import subgraphmatchgpu_b200 as sme
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [sme.EXT_CACHE, sme.EXT_UMA])
def test_external_mode_matches_reference(golden, variant):
    for name in ("rmat_s12_ef8", "ba_n600_m4"):
        g = sme.Graph.load(golden_graph_path(name))
        for q, want in golden[name]["counts"].items():
            if int(want) > 3_000_000_000:
                continue
            got = g.count(int(q), sme.GPU_LIGHT, sme.EXTERNAL_GPU, ext_variant=variant)
            assert got == want, (name, q, variant)


def test_external_mode_small_budget_loads_many_subgraphs(golden):
    # many batches, and every adjacency list crosses the host link at most
    # once: lists loaded for one batch stay in the device list cache for the
    # next batches and steps (incremental loading)
    g = sme.Graph.load(golden_graph_path("rmat_s12_ef8"))
    n, m, _ = g.info()
    for q in (0, 3, 4, 1):
        got = g.count(q, sme.GPU_LIGHT, sme.EXTERNAL_GPU, mem_limit_bytes=16 << 20)
        assert got == golden["rmat_s12_ef8"]["counts"][str(q)]
        s = sme.last_stats()
        assert s.batches > 2
        assert 8 * (n + 1) < s.h2d_bytes <= 8 * (n + 1) + 4 * m


def test_external_mode_restarts_its_list_cache():
    # R-MAT s16 ef16 holds ~7 MB of lists; a 12 MiB budget leaves the list
    # cache about 6 MB of it, so it fills and starts over while sets computed
    # earlier (copies, never views into the cache) live on
    g = sme.Graph.rmat(16, 16, seed=3)
    n, m, _ = g.info()
    assert 4 * m > 6.5 * (1 << 20)
    for q in (0, 3, 2, 1):
        want = g.count(q, sme.GPU_LIGHT, root_stride=7 if q == 1 else 1)
        try:
            got = g.count(q, sme.GPU_LIGHT, sme.EXTERNAL_GPU, mem_limit_bytes=12 << 20,
                          root_stride=7 if q == 1 else 1)
        except sme.SmeError as e:
            raise AssertionError(f"Q{q}: {e}")
        assert got == want, q
        s = sme.last_stats()
        assert s.batches > 2 and s.h2d_bytes > 8 * (n + 1)


def small_graphs(num, seed):
    rnd = random.Random(seed)
    gs, qs = [], []
    for i in range(num):
        n = int(round(2 ** rnd.uniform(6, 10)))  # 64 .. 1024 (log-uniform)
        d = rnd.uniform(4, 32)
        if i % 2 == 0:
            g = sme.Graph.er(n, d, seed=seed * 10007 + i)
        else:
            g = sme.Graph.ba(n, max(1, int(round(d / 2))), seed=seed * 10007 + i)
        gs.append(g)
        qs.append(rnd.choice([0, 1, 2, 3]))
    return gs, qs


def test_batched_form_matches_oracle_per_graph():
    gs, qs = small_graphs(96, 5)
    want = np.array([O.count(*g.csr(), q) for g, q in zip(gs, qs)], dtype=np.uint64)
    plan = sme.BatchPlan(gs, qs, autotune=True, use_graph=True)
    got, ms = plan.run()
    assert np.array_equal(got, want)
    got2, _ = plan.run()  # graph replay
    assert np.array_equal(got2, want)
    d = plan.describe()
    assert d["group_threads"] in (4, 8, 16, 32, 64, 128) and d["work_items"] == sum(g.n for g in gs)
    assert d["items_per_fetch"] in (1, 4, 16) and d["tuned_ms"] > 0


@pytest.mark.parametrize("gran,block", [(0, 128), (1, 128), (2, 256), (2, 128)])
def test_batched_form_fixed_configurations(gran, block):
    # 0: eight lanes, 1: a warp, 2: a CTA group of 128 threads per item
    gs, qs = small_graphs(40, 9)
    want = np.array([O.count(*g.csr(), q) for g, q in zip(gs, qs)], dtype=np.uint64)
    plan = sme.BatchPlan(gs, qs, autotune=False, use_graph=False, granularity=gran, block_threads=block)
    got, _ = plan.run()
    assert np.array_equal(got, want)
    assert plan.describe()["group_threads"] == {0: 8, 1: 32, 2: 128}[gran]


def test_batched_form_all_queries():
    gs = [sme.Graph.er(80, 10.0, seed=s) for s in range(14)]
    qs = list(range(14))
    want = np.array([O.count(*g.csr(), q) for g, q in zip(gs, qs)], dtype=np.uint64)
    got, _ = sme.BatchPlan(gs, qs).run()
    assert np.array_equal(got, want)


def test_served_form_results_same_alone_and_in_mix():
    big = sme.Graph.rmat(12, 8, seed=3)
    mid = sme.Graph.rmat(10, 8, seed=4)
    srv = sme.Server(slots=4)
    gids = [srv.add_graph(big), srv.add_graph(mid)]
    attached = [sme.Graph.er(n, 8.0, seed=n) for n in (256, 1024, 4096)]
    reqs = []
    rnd = random.Random(1)
    for i in range(30):
        q = rnd.choice([0, 1, 2, 3, 4, 7])
        if i % 3 == 2:
            reqs.append((q, -1, attached[i % 3]))
        else:
            reqs.append((q, gids[i % 2], None))
    # alone: one at a time
    alone = []
    for q, gid, att in reqs:
        alone.append(srv.wait(srv.submit(q, gid=gid, attached=att))[0])
    # in the mix: all submitted at once
    ids = [srv.submit(q, gid=gid, attached=att) for q, gid, att in reqs]
    mixed = [srv.wait(i)[0] for i in ids]
    assert mixed == alone
    # and both equal the oracle
    graphs = {gids[0]: big, gids[1]: mid}
    for (q, gid, att), c in zip(reqs, alone):
        g = att if att is not None else graphs[gid]
        assert c == O.count(*g.csr(), q)
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["max_inflight"] >= 2
    srv.close()


def test_served_form_rejects_bad_requests():
    srv = sme.Server(slots=2)
    g = sme.Graph.clique(6)
    gid = srv.add_graph(g)
    with pytest.raises(sme.SmeError):
        srv.submit(14, gid=gid)
    with pytest.raises(sme.SmeError):
        srv.submit(0, gid=7)
    assert srv.wait(srv.submit(3, gid=gid))[0] == 15
    srv.close()
