"""The drop-in `patternmatchgpu` binary: the reference's flags and result line."""
import os
import re
import subprocess

import pytest

from conftest import ROOT, golden_graph_path

BIN = os.path.join(ROOT, "subgraphmatchgpu_b200", "bin", "patternmatchgpu")


def run(*args):
    return subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=300)


def test_help_without_arguments():
    r = run()
    assert r.returncode == 255
    assert "ALGORITHM: ,GPU_GPSM=4,GPU_GPSM_REUSE=5,GPU_LIGHT=6" in r.stdout
    assert "DEGREE_ORDER" in r.stdout


def test_rejects_partitioned_and_bad_degree_order():
    g = golden_graph_path("k12")
    r = run("-f", g, "-d", 0, "-a", 6, "-q", 3, "-m", 1, "-p", 2)
    assert r.returncode == 1 and "-m 0" in r.stderr
    r = run("-f", g, "-d", 0, "-a", 6, "-q", 3, "-m", 1, "-O", 5)
    assert r.returncode == 1 and "-O" in r.stderr


def test_oriented_graph_rejects_non_clique_query():
    r = run("-f", golden_graph_path("k12"), "-d", 0, "-a", 6, "-q", 1, "-m", 1, "-O", 2)
    assert r.returncode == 1
    assert "status 6" in r.stderr and "clique" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("order", [0, 1, 2])
def test_result_line_matches_reference_count(golden, order):
    name = "rmat_s10_ef8"
    for q in (0, 3, 7):
        r = run("-f", golden_graph_path(name), "-d", 0, "-a", 6, "-q", q, "-m", 1, "-O", order)
        assert r.returncode == 0, r.stderr
        m = re.search(r"^total_match_count=(\d+), elapsed_time=([0-9.e+-]+)ms$", r.stdout, re.M)
        assert m and int(m.group(1)) == golden[name]["counts"][str(q)], r.stdout


def test_hybrid_mode_checks_the_partition_file(tmp_path):
    g = golden_graph_path("k12")
    short = tmp_path / "short.part.2"
    short.write_text("0\n1\n0\n")
    r = run("-f", g, "-d", 0, "-a", 6, "-q", 3, "-m", 0, "-e", short, "-p", 2)
    assert r.returncode == 1 and "partition file" in r.stderr and "ends after 3 of 12" in r.stderr
    # the reference runs -m 0 with the reuse BFS or LIGHT plan only
    ok = tmp_path / "k12.part.2"
    ok.write_text("\n".join(str(i % 2) for i in range(12)))
    r = run("-f", g, "-d", 0, "-a", 4, "-q", 3, "-m", 0, "-e", ok, "-p", 2)
    assert r.returncode == 1 and "reuse BFS (5) or LIGHT (6)" in r.stderr


@pytest.mark.gpu
def test_hybrid_mode_result_lines(golden, tmp_path):
    name = "rmat_s10_ef8"
    n = 797
    part = tmp_path / "g.part.3"
    part.write_text("\n".join(str((i * 7) % 3) for i in range(n)))
    r = run("-f", golden_graph_path(name), "-d", 0, "-a", 6, "-q", 3, "-m", 0, "-e", part, "-p", 3)
    assert r.returncode == 0, r.stderr
    intra = [int(x) for x in re.findall(r"^partition_id=\d+,intra_partition_count=(\d+)$", r.stdout, re.M)]
    inter = int(re.search(r"^inter_partition_count=(\d+)$", r.stdout, re.M).group(1))
    total = int(re.search(r"^total_match_count=(\d+), elapsed_time=", r.stdout, re.M).group(1))
    assert len(intra) == 3 and total == golden[name]["counts"]["3"] and sum(intra) + inter == total


def test_preprocess_graph_tool_writes_what_the_reference_tool_writes(tmp_path):
    # same flags and output names as the reference's preprocess_graph; the
    # hashes were taken from the reference tool (tests/golden/make_golden.py)
    import hashlib
    import json
    import shutil
    tool = os.path.join(ROOT, "subgraphmatchgpu_b200", "bin", "preprocess_graph")
    golden = os.path.join(ROOT, "tests", "golden")
    pre = json.load(open(os.path.join(golden, "preprocess.json")))
    fmt = json.load(open(os.path.join(golden, "formats.json")))
    txt = tmp_path / "messy.txt"
    shutil.copy(os.path.join(golden, "messy_edges.txt"), txt)
    lvid = tmp_path / "messy.lvid"
    shutil.copy(os.path.join(golden, "messy.lvid"), lvid)

    def sha(p):
        return hashlib.sha256(open(p, "rb").read()).hexdigest()

    for args, out, want in (((txt, 1), str(txt) + ".bin", pre["reference_sha256"]),
                            ((txt, 0), str(txt) + ".snap.txt", fmt["reference.snap.txt"]),
                            ((txt, 3), str(txt) + ".adj.txt", fmt["reference.adj.txt"]),
                            ((lvid, 1), str(lvid) + ".bin", fmt["reference.lvid.bin"])):
        r = subprocess.run([tool, "-f", str(args[0]), "-d", "0", "-o", str(args[1])], capture_output=True,
                           text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        assert sha(out) == want, out
    assert open(str(txt) + ".adj.txt.info").read() == fmt["reference.adj.txt.info"]
