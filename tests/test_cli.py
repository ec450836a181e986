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
    assert r.returncode == 1 and "-p 1" in r.stderr
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
