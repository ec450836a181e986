"""Host-side logic of libsme without a GPU: the C-ABI surface, formats,
preprocessing, generators and the three query plans."""
import hashlib
import json
import os
import re

import numpy as np
import pytest

import subgraphmatchgpu_b200 as sme
from conftest import ROOT, golden_graph_path

HEADER = os.path.join(ROOT, "include", "sme.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sme_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = sme.lib()
    names = header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in sme.SIGNATURES, f"{n} missing from the Python signature table"


def test_version_and_opts_defaults():
    assert b"sm_100a" in sme.lib().sme_version()
    o = sme.opts(3)
    assert (o.algo, o.execute_mode, o.compress_level, o.enable_ordering) == (6, 1, 3, 1)


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_bin_roundtrip_is_byte_identical(tmp_path, golden):
    for name in ("k6", "rmat_s10_ef8", "ba_n600_m4"):
        g = sme.Graph.load(golden_graph_path(name))
        out = str(tmp_path / "x.bin")
        g.write_bin(out)
        assert sha(out) == golden[name]["sha256"]
        g.validate()


def test_generators_are_deterministic(golden):
    g = sme.Graph.rmat(10, 8, seed=12)
    n, m, d = g.info()
    assert (n, m, d) == (golden["rmat_s10_ef8"]["n"], golden["rmat_s10_ef8"]["m"], golden["rmat_s10_ef8"]["max_degree"])
    g.validate()
    g2 = sme.Graph.rmat(10, 8, seed=12)
    for a, b in zip(g.csr(), g2.csr()):
        assert np.array_equal(a, b)
    for h in (sme.Graph.er(300, 6.0, seed=3), sme.Graph.ba(300, 3, seed=3), sme.Graph.clique(7)):
        h.validate()


def test_preprocess_matches_reference_preprocess_graph(tmp_path):
    rec = json.load(open(os.path.join(ROOT, "tests", "golden", "preprocess.json")))
    g = sme.Graph.load(os.path.join(ROOT, "tests", "golden", "messy_edges.txt"), 0)
    g.preprocess()
    out = str(tmp_path / "m.bin")
    g.write_bin(out)
    assert sha(out) == rec["reference_sha256"] == rec["libsme_sha256"]


def test_bad_inputs_return_status(tmp_path):
    p = tmp_path / "trunc.bin"
    p.write_bytes(b"\x04" + b"\x00" * 20)
    with pytest.raises(sme.SmeError) as e:
        sme.Graph.load(str(p))
    assert e.value.status == 2
    src = open(golden_graph_path("k6"), "rb").read()
    p.write_bytes(src[:-3])
    with pytest.raises(sme.SmeError):
        sme.Graph.load(str(p))
    p.write_bytes(src[:8] + (5).to_bytes(8, "little") + src[16:])  # uintE size 5
    with pytest.raises(sme.SmeError):
        sme.Graph.load(str(p))
    with pytest.raises(sme.SmeError):
        sme.Graph.load(str(tmp_path / "missing.bin"))
    with pytest.raises(sme.SmeError) as e:
        sme.plan_describe(14, 2)
    assert e.value.status == 6
    with pytest.raises(sme.SmeError):
        sme.Graph.from_csr(np.array([0, 2, 1], np.uint64), np.array([1, 0], np.uint32))
    with pytest.raises(sme.SmeError):
        sme.Graph.from_csr(np.array([0, 1, 2], np.uint64), np.array([1, 5], np.uint32))


@pytest.mark.parametrize("q", range(14))
def test_light_plan_matches_reference_test_plan(q):
    ref = open(os.path.join(ROOT, "tests", "golden", "plans", f"q{q}_light_nonmat_opt.txt")).read()
    block = ref.split(f"Lazy traversal plan for Q{q}--------------------\n")[1].split("-----")[0]
    mine = sme.plan_describe(q, 2).strip().splitlines()[1:]
    assert block.strip().splitlines() == mine


@pytest.mark.parametrize("q", range(14))
def test_reuse_autogen_plan_matches_reference_test_plan(q):
    ref = open(os.path.join(ROOT, "tests", "golden", "plans", f"q{q}_reuse_autogen.txt")).read()
    rl = [l for l in ref.splitlines() if l.startswith("level ")]
    ml = [l.split("  (cached)")[0] for l in sme.plan_describe(q, 1).splitlines() if l.startswith("level ")]
    assert rl == ml


HARDCODED = (0, 2, 3, 5, 6, 7, 8, 9, 10, 11, 12, 13)


@pytest.mark.parametrize("q", HARDCODED)
def test_hardcoded_reuse_plan_matches_reference(q):
    # the plan `patternmatchgpu -a 5` runs: search sequence, per-level reuse
    # metas and separate lists, and every meta's vertex mapping
    ref = open(os.path.join(ROOT, "tests", "golden", "plans", f"q{q}_reuse_hardcoded.txt")).read().splitlines()
    mine = sme.plan_describe(q, 3).splitlines()
    rl = [l for l in ref if l.startswith(("level ", "mapping level "))]
    ml = [l.split("  (cached)")[0] for l in mine if l.startswith(("level ", "mapping level "))]
    assert rl == ml
    seq = next(l for l in ref if l.startswith("search sequence for intra-partition:")).split(":")[1].split()
    assert mine[0].split("search sequence:")[1].split() == seq


def test_special_plans_and_hardcoded_reuse():
    # COMPRESS_LEVEL_SPECIAL (LazyTraversalPlanGenerator.h:244-300)
    q2 = sme.plan_describe(2, 4)
    assert "(COMPUTE_PATH_COUNT,1),(COMPUTE_PATH_COUNT,3),(COUNT,4)" in q2
    assert "(COUNT,6)" in sme.plan_describe(5, 4)
    # hard-coded reuse plans exist for every query but Q1/Q4
    for q in HARDCODED:
        sme.plan_describe(q, 3)
    for q in (1, 4):
        with pytest.raises(sme.SmeError) as e:
            sme.plan_describe(q, 3)
        assert e.value.status == 6
    q7 = sme.plan_describe(7, 3)
    assert "level 4, vertex=4:intersect: [source_vertex=3,conn=(0,1,2),source_conn=(0,1,2)] 3" in q7


def test_compiled_programs_are_consistent():
    for q in range(14):
        text = sme.plan_describe(q, 5)
        assert text.count("program Q") == 3
        # every program starts with the roots and ends in a counting step
        for prog in text.split("program Q")[1:]:
            lines = prog.strip().splitlines()[1:]
            assert lines[0].split(":")[1].strip().startswith("INIT")
            assert re.search(r"(COMPUTE_COUNT|COUNT)\(", lines[-1])


CLIQUES = (0, 3, 7, 11)


def test_degree_order_is_an_isomorphism_sorted_by_degree():
    g = sme.Graph.rmat(10, 8, seed=5)
    rp, cl = g.csr()
    d, new_to_old = g.degree_order()
    assert not d.oriented
    drp, dcl = d.csr()
    n = len(rp) - 1
    assert len(drp) == n + 1 and len(dcl) == len(cl)
    assert sorted(new_to_old.tolist()) == list(range(n))
    deg_old, deg_new = np.diff(rp).astype(np.int64), np.diff(drp).astype(np.int64)
    assert np.array_equal(deg_new, deg_old[new_to_old])
    keys = deg_new.astype(np.int64) * n + new_to_old.astype(np.int64)
    assert np.all(np.diff(keys) > 0)  # (degree, original id) ascending
    d.validate()
    old_edges = set(zip(np.repeat(np.arange(n), deg_old).tolist(), cl.tolist()))
    new_edges = zip(new_to_old[np.repeat(np.arange(n), deg_new)].tolist(), new_to_old[dcl].tolist())
    assert set(new_edges) == old_edges


@pytest.mark.parametrize("name", ["rmat_s10_ef8", "ba_n600_m4", "er_n64_d12"])
def test_degree_order_preserves_every_count(golden, name):
    import oracle_py as O
    rp, cl = O.read_bin(golden_graph_path(name))
    d, _ = sme.Graph.from_csr(rp, cl).degree_order()
    drp, dcl = d.csr()
    for q, want in golden[name]["counts"].items():
        if want > 5e7:
            continue
        assert O.count(drp, dcl, int(q)) == want, (name, q)


def test_oriented_graph_keeps_each_edge_once_towards_higher_id():
    g = sme.Graph.rmat(10, 8, seed=5)
    _, cl = g.csr()
    o, _ = g.degree_order(orient=True)
    assert o.oriented
    orp, ocl = o.csr()
    assert 2 * len(ocl) == len(cl)
    src = np.repeat(np.arange(len(orp) - 1), np.diff(orp).astype(np.int64))
    assert np.all(ocl > src)
    with pytest.raises(sme.SmeError) as e:
        o.preprocess()
    assert e.value.status == 1
    with pytest.raises(sme.SmeError) as e:
        o.degree_order()
    assert e.value.status == 1


@pytest.mark.parametrize("q", [1, 2, 4, 5, 6, 8, 9, 10, 12, 13])
def test_oriented_graph_rejects_non_clique_queries(q):
    # checked at plan time, before any device call
    o, _ = sme.Graph.rmat(8, 8, seed=2).degree_order(orient=True)
    for algo in (4, 5, 6):
        with pytest.raises(sme.SmeError) as e:
            o.count(q, algo)
        assert e.value.status == 6, (q, algo)
    with pytest.raises(sme.SmeError) as e:
        o.count(3, 6, enable_ordering=0)
    assert e.value.status == 6


def test_clique_plans_read_lists_along_the_orientation():
    # every clique plan (all three algorithms, every LIGHT compress level)
    # passes the plan-time orientation check: the count on an oriented graph
    # reaches the device stage (without a GPU: a device error, not status 6)
    o, _ = sme.Graph.rmat(8, 8, seed=2).degree_order(orient=True)
    for q in CLIQUES:
        for algo, kw in ((4, {}), (5, {}), (5, {"reuse_autogen": 1})) + tuple((6, {"compress_level": c})
                                                                           for c in range(4)):
            try:
                o.count(q, algo, **kw)
            except sme.SmeError as e:
                assert e.status != 6, (q, algo, kw, str(e))


def test_light_clique_programs_start_from_earlier_sets():
    # 4-clique: the count step intersects set(2) = N(0) ∩ N(1) ∩ {> 1} with
    # N(2) instead of three lists; set(2) stays with the children of M(2)
    light = sme.plan_describe(3, 5).split("program Q")[3]
    assert "MATERIALIZE(2) keep" in light
    # the != conditions the total order implies are dropped
    assert "COMPUTE_COUNT(3) conn=(2) reuse=2 cond=(>2)" in light
    # 4-cycle: no earlier set covers two of its lists; u2 != u1 is a real check
    q1 = sme.plan_describe(1, 5).split("program Q")[3]
    assert "reuse=" not in q1
    assert "COMPUTE(2) conn=(1) cond=(>0,!=1)" in q1
    # without self loops a candidate from N(M[v]) differs from M[v]: the
    # 4-cycle keeps only its order conditions
    q1 = sme.plan_describe(1, 6).split("program Q")[3]
    assert "COMPUTE(2) conn=(1) cond=(>0)" in q1
    assert "COMPUTE_COUNT(3) conn=(0,2) cond=(>0,>1)" in q1
    # a != against a vertex that is not a list owner stays (house: u4 vs u1)
    assert "!=" in sme.plan_describe(4, 6).split("program Q")[3]


def test_partition_file_reader(tmp_path):
    f = tmp_path / "g.part.3"
    f.write_text("0 1 2\n2 1\n0\n")
    assert sme.read_partition_file(str(f), 6, 3).tolist() == [0, 1, 2, 2, 1, 0]
    # one partition (or no file): everything in partition 0
    assert sme.read_partition_file("", 4, 1).tolist() == [0, 0, 0, 0]
    for text, n, k in (("0 1\n", 3, 2), ("0 3 1\n", 3, 3), ("0 1 1\n", 3, 3)):
        f.write_text(text)
        with pytest.raises(sme.SmeError) as e:
            sme.read_partition_file(str(f), n, k)
        assert e.value.status == 2, text


def test_induced_partition_subgraph():
    import oracle_py as O
    g = sme.Graph.rmat(10, 8, seed=9)
    rp, cl = g.csr()
    n = len(rp) - 1
    part = (np.arange(n) * 5 % 3).astype(np.uint32)
    for p in range(3):
        sub = g.partition(part, p)
        srp, scl = sub.csr()
        members = np.flatnonzero(part == p)
        local = {int(v): i for i, v in enumerate(members)}
        want_edges = sorted((local[int(u)], local[int(v)]) for u in members
                            for v in cl[rp[u]:rp[u + 1]] if part[v] == p)
        got_edges = sorted(zip(np.repeat(np.arange(len(srp) - 1), np.diff(srp).astype(np.int64)).tolist(),
                               scl.tolist()))
        assert len(srp) - 1 == len(members) and got_edges == want_edges
        # the induced subgraph keeps exactly the instances inside the partition
        inst = O.enumerate_sorted(rp, cl, 3)
        inside = int(np.all(part[inst] == p, axis=1).sum())
        assert O.count(srp, scl, 3) == inside
    with pytest.raises(sme.SmeError) as e:
        g.count_partitioned(3, part, 3, algo=sme.GPU_GPSM)
    assert e.value.status == 1


@pytest.mark.parametrize("plan_type", [5, 6])
def test_reused_sets_are_live_where_they_are_read(plan_type):
    # every step that starts from an earlier candidate set must find that set
    # among the live sets left by the step before it, and every list it
    # reads must belong to a vertex materialised by then
    step_re = re.compile(r"^(\d+): (\w+)\((\d+)\)(.*)\| mat=\(([\d,]*)\) sets=\(([\d,]*)\)$")
    for q in range(14):
        for prog in sme.plan_describe(q, plan_type).split("program Q")[1:]:
            live, mat = set(), set()
            for line in prog.strip().splitlines()[1:]:
                m = step_re.match(line.strip())
                assert m, line
                kind, u, rest = m.group(2), int(m.group(3)), m.group(4)
                r = re.search(r"reuse=(\d+)", rest)
                if r:
                    assert int(r.group(1)) in live, (q, plan_type, line)
                c = re.search(r"conn=\(([\d,]+)\)", rest)
                if c:
                    assert {int(x) for x in c.group(1).split(",")} <= mat, (q, plan_type, line)
                mat = {int(x) for x in m.group(5).split(",") if x}
                live = {int(x) for x in m.group(6).split(",") if x}


def test_snap_adj_and_lvid_formats_match_reference_preprocess_graph(tmp_path):
    # pinned by tests/golden/make_golden.py against the reference's
    # preprocess_graph (-o 0 SNAP text, -o 3 ADJ text + info, .lvid input)
    rec = json.load(open(os.path.join(ROOT, "tests", "golden", "formats.json")))
    g = sme.Graph.load(os.path.join(ROOT, "tests", "golden", "messy_edges.txt"), 0)
    g.preprocess()
    g.write_snap(str(tmp_path / "g.snap"))
    g.write_adj(str(tmp_path / "g.adj"))
    assert sha(str(tmp_path / "g.snap")) == rec["reference.snap.txt"]
    assert sha(str(tmp_path / "g.adj")) == rec["reference.adj.txt"]
    assert (tmp_path / "g.adj.info").read_text() == rec["reference.adj.txt.info"]
    lv = sme.Graph.load(os.path.join(ROOT, "tests", "golden", "messy.lvid"), 0)
    lv.preprocess()
    lv.write_bin(str(tmp_path / "lvid.bin"))
    assert sha(str(tmp_path / "lvid.bin")) == rec["reference.lvid.bin"]


def test_lvid_names_are_exact_strings(tmp_path):
    f = tmp_path / "x.lvid"
    f.write_text("# names\n7 007\n007 123456789012345\n123456789012345,7\n")
    g = sme.Graph.load(str(f), 0)
    # 7 -> 0, 007 -> 1, 123456789012345 -> 2: a triangle
    assert g.info()[:2] == (3, 6)
    rp, cl = g.csr()
    assert rp.tolist() == [0, 2, 4, 6] and cl.tolist() == [1, 2, 0, 2, 0, 1]
    f.write_text("1 2 3\n")
    with pytest.raises(sme.SmeError) as e:
        sme.Graph.load(str(f), 0)
    assert e.value.status == 2


def test_pack_reports_the_bytes_an_upload_copies():
    g = sme.Graph.rmat(12, 8, seed=3)
    plain = (g.n + 1) * 8 + g.m * 4
    b = g.pack()
    assert 0 < b < 0.7 * plain
    assert g.pack() == b  # deterministic
    assert g.pack(False) == 0
    with pytest.raises(sme.SmeError) as e:
        g.device_arrays(0)
    assert e.value.status == 1
