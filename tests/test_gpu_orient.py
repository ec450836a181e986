"""Degree-ordered and oriented graphs on the GPU: a renumbering preserves every
count; an oriented graph (each edge once, towards the higher id) preserves
the clique counts under every plan, mode and form, and rejects the rest."""
import numpy as np
import pytest

import oracle_py as O
import subgraphmatchgpu_b200 as sme
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu

ALGOS = (sme.GPU_GPSM, sme.GPU_GPSM_REUSE, sme.GPU_LIGHT)
CLIQUES = (0, 3, 7, 11)
GPU_LIMIT = 3_000_000_000


@pytest.fixture(scope="module")
def ordered(golden):
    out = {}
    for name in golden:
        g = sme.Graph.load(golden_graph_path(name))
        d, _ = g.degree_order()
        o, m = g.degree_order(orient=True)
        out[name] = (d, o, m)
    return out


def test_degree_ordered_counts_match_reference(ordered, golden):
    for name, d in golden.items():
        g = ordered[name][0]
        for q, want in d["counts"].items():
            if want > GPU_LIMIT:
                continue
            for algo in ALGOS:
                assert g.count(int(q), algo) == want, (name, q, algo)


def test_oriented_clique_counts_match_reference(ordered, golden):
    for name, d in golden.items():
        o = ordered[name][1]
        for q in CLIQUES:
            want = d["counts"].get(str(q))
            if want is None or want > GPU_LIMIT:
                continue
            for algo in ALGOS:
                assert o.count(q, algo) == want, (name, q, algo)
            for level in range(4):
                assert o.count(q, sme.GPU_LIGHT, compress_level=level) == want, (name, q, level)
            assert o.count(q, sme.GPU_GPSM_REUSE, reuse_autogen=1) == want, (name, q)
            for variant in (sme.EXT_CACHE, sme.EXT_UMA):
                got = o.count(q, sme.GPU_LIGHT, mode=sme.EXTERNAL_GPU, ext_variant=variant)
                assert got == want, (name, q, variant)


@pytest.mark.parametrize("name", ["er_n64_d12", "k12", "rmat_s8_ef8"])
def test_oriented_instances_map_back_to_the_same_vertex_sets(ordered, name):
    rp, cl = O.read_bin(golden_graph_path(name))
    o, new_to_old = ordered[name][1], ordered[name][2]
    for q in (0, 3, 7):
        want = O.sort_rows(np.sort(O.enumerate_sorted(rp, cl, q), axis=1))
        for algo in ALGOS:
            got = o.enumerate(q, algo)
            got = O.sort_rows(np.sort(new_to_old[got], axis=1))
            assert np.array_equal(got, want), (name, q, algo)


def test_oriented_batched_and_served_forms():
    gs = [sme.Graph.er(n, 12.0, seed=n).degree_order(orient=True)[0] for n in (64, 200, 700, 1500)]
    src = [sme.Graph.er(n, 12.0, seed=n) for n in (64, 200, 700, 1500)]
    qs = [0, 3, 7, 3]
    want = np.array([O.count(*g.csr(), q) for g, q in zip(src, qs)], dtype=np.uint64)
    got, _ = sme.BatchPlan(gs, qs).run()
    assert np.array_equal(got, want)
    with pytest.raises(sme.SmeError) as e:
        sme.BatchPlan(gs, [0, 1, 7, 3])
    assert e.value.status == 6
    srv = sme.Server(slots=2)
    gid = srv.add_graph(gs[3])
    assert srv.wait(srv.submit(3, gid=gid))[0] == want[3]
    assert srv.wait(srv.submit(7, gid=gid, algo=sme.GPU_GPSM_REUSE))[0] == O.count(*src[3].csr(), 7)
    with pytest.raises(sme.SmeError) as e:
        srv.wait(srv.submit(2, gid=gid))
    assert e.value.status == 6
    srv.close()
