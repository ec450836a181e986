"""The bench's workload on CPU: the numpy R-MAT edge list reaches the same CSR
through the engine's preprocessing, the oracle's and the reference's own
preprocess_graph; both arms build the same step list and configuration; the
reference's CPU_WCOJ task driver agrees with the oracle on those steps."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import oracle_py as O

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
need_ref = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "ref_wcoj_task")),
                              reason="reference tools not built (make -C oracle ref)")


def small_args(*extra):
    return bench.parse(["--scale", "12", "--edge-factor", "8", "--blocks", "3:512,1:64,2:256", *extra])


def test_rmat_edges_are_seeded_and_in_range():
    u1, v1 = bench.rmat_edges(10, 4, seed=3)
    u2, v2 = bench.rmat_edges(10, 4, seed=3)
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)
    assert len(u1) == 4096 and u1.max() < 1024 and v1.max() < 1024
    u3, _ = bench.rmat_edges(10, 4, seed=4)
    assert not np.array_equal(u1, u3)
    # a = .57 puts most edges in the top-left quadrant: low ids dominate
    assert (u1 < 512).mean() > 0.7


def test_engine_and_oracle_preprocessing_agree():
    import subgraphmatchgpu_b200 as sme
    args = small_args()
    g = bench.engine_graph(args)
    u, v = bench.rmat_edges(args.scale, args.edge_factor, seed=args.seed)
    rp, cl = O.preprocess_csr(*bench.raw_csr(u, v, 1 << args.scale))
    erp, ecl = g.csr()
    assert np.array_equal(rp, erp) and np.array_equal(cl, ecl)
    sme.Graph.from_csr(rp, cl).validate()


@need_ref
def test_reference_preprocess_tool_gives_the_same_bin():
    args = small_args()
    with tempfile.TemporaryDirectory() as tmp:
        bin_path, rp, cl = bench.reference_graph(args, tmp)
        assert bin_path is not None
    g = bench.engine_graph(args)
    erp, ecl = g.csr()
    assert np.array_equal(rp, erp) and np.array_equal(cl, ecl)


def test_step_list_is_deterministic_and_avoids_hubs():
    args = small_args()
    g = bench.engine_graph(args)
    rp, _ = g.csr()
    a = bench.make_steps(rp, args, 9)
    b = bench.make_steps(rp, args, 9)
    deg = np.diff(rp)
    assert [q for q, _ in a] == [3, 1, 2] * 3
    for (qa, ra), (qb, rb) in zip(a, b):
        assert qa == qb and np.array_equal(ra, rb)
        assert len(ra) == {3: 512, 1: 64, 2: 256}[qa]
        assert (deg[ra] <= args.hub_degree).all()
    # consecutive blocks of one query are disjoint until the pool wraps
    q3 = [r for q, r in a if q == 3]
    assert not set(q3[0].tolist()) & set(q3[1].tolist())


@need_ref
def test_reference_task_driver_matches_oracle_on_the_steps():
    args = small_args()
    with tempfile.TemporaryDirectory() as tmp:
        bin_path, rp, cl = bench.reference_graph(args, tmp)
        steps = bench.make_steps(rp, args, 6)
        ref = bench.reference_tasks(bin_path, steps, 4, tmp)
    port = bench.port_tasks(rp, cl, steps, 4)
    assert [c for c, _ in ref] == [c for c, _ in port]
    assert all(c > 0 for c, _ in ref)


@need_ref
def test_reference_task_driver_strided_tasks():
    rp, cl = O.read_bin(os.path.join(ROOT, "tests", "golden", "graphs", "rmat_s12_ef8.bin"))
    r = subprocess.run([os.path.join(REF, "ref_wcoj_task"), "-f",
                        os.path.join(ROOT, "tests", "golden", "graphs", "rmat_s12_ef8.bin"), "-q", "3", "-t", "2",
                        "S:4:1", "S:1:0"], capture_output=True, text=True, check=True)
    got = [int(dict(x.strip().split("=", 1) for x in ln.split(","))["total_match_count"])
           for ln in r.stdout.splitlines() if ln.startswith("task=")]
    assert got == [O.count_strided(rp, cl, 3, 4, 1), O.count(rp, cl, 3)]


def test_both_arms_print_the_same_config():
    args = small_args()
    g = bench.engine_graph(args)
    rp, cl = g.csr()
    a = bench.config_of(args, len(rp) - 1, len(cl), bench.csr_digest(rp, cl))
    u, v = bench.rmat_edges(args.scale, args.edge_factor, seed=args.seed)
    rrp, rcl = O.preprocess_csr(*bench.raw_csr(u, v, 1 << args.scale))
    b = bench.config_of(args, len(rrp) - 1, len(rcl), bench.csr_digest(rrp, rcl))
    assert a == b


def test_reference_arm_port_fallback(monkeypatch, capsys):
    # without the reference's tools the arm times the oracle's restatement on
    # the same steps and says so
    import json
    monkeypatch.setattr(bench, "REF_TASK", "/nonexistent/ref_wcoj_task")
    args = small_args("--impl", "reference", "--steps", "3", "--warmup", "0")
    bench.run_reference(args, 0, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["cpu_baseline"]["kind"] == "port"
    steps = bench.make_steps(bench.engine_graph(args).csr()[0], args, 3)
    rp, cl = bench.engine_graph(args).csr()
    assert line["step_counts"] == [O.count_roots(rp, cl, q, r) for q, r in steps]
