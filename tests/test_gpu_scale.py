"""R-MAT scale 22, edge factor 16 (the 5-clique / house configuration):
size-independent properties at full size.

* 4-clique on the degree-ordered oriented graph: LIGHT, reuse-BFS and plain
  BFS agree, and equal the count on the original graph.
* 5-clique on the oriented graph, every 256th root: the three plans, LIGHT
  without set reuse and LIGHT in external mode (lists gathered from host
  memory) agree root task by root task (all plans root at pattern vertex 0).
* house on the original graph, every 65536th root from 1000003: LIGHT in memory and in
  both external variants agree, with and without set reuse.
"""
import pytest

import subgraphmatchgpu_b200 as sme

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s22():
    g = sme.Graph.rmat(22, 16, seed=22)
    o, _ = g.degree_order(orient=True)
    o.to_device(0)
    yield g, o
    o.release_device()


def test_four_clique_full_graph(s22):
    g, o = s22
    light = o.count(3, sme.GPU_LIGHT)
    assert light > 10 ** 11
    assert o.count(3, sme.GPU_GPSM_REUSE) == light
    assert o.count(3, sme.GPU_GPSM) == light
    g.to_device(0)
    try:
        assert g.count(3, sme.GPU_GPSM_REUSE) == light
    finally:
        g.release_device()


def test_five_clique_root_sample(s22):
    _, o = s22
    kw = dict(root_stride=256, root_begin=7)
    light = o.count(7, sme.GPU_LIGHT, **kw)
    assert light > 0
    assert o.count(7, sme.GPU_GPSM_REUSE, **kw) == light
    assert o.count(7, sme.GPU_GPSM, **kw) == light
    assert o.count(7, sme.GPU_LIGHT, no_set_reuse=1, **kw) == light
    assert o.count(7, sme.GPU_LIGHT, mode=sme.EXTERNAL_GPU, **kw) == light


def test_house_root_sample(s22):
    g, _ = s22
    kw = dict(root_stride=65536, root_begin=1_000_003)
    g.to_device(0)
    try:
        light = g.count(4, sme.GPU_LIGHT, **kw)
        assert light > 0
        assert g.count(4, sme.GPU_LIGHT, no_set_reuse=1, **kw) == light
    finally:
        g.release_device()
    for variant in (sme.EXT_CACHE, sme.EXT_UMA):
        assert g.count(4, sme.GPU_LIGHT, mode=sme.EXTERNAL_GPU, ext_variant=variant, **kw) == light
