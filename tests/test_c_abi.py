"""The C ABI from a plain C99 caller: include/sme.h compiles as C, libsme.so
links and its host-side entry points answer (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT, golden_graph_path

C_SRC = r"""
#include <stdio.h>
#include <stdlib.h>
#include "sme.h"

int main(int argc, char** argv) {
  sme_graph* g = NULL;
  uint64_t n = 0, m = 0, d = 0;
  if (sme_graph_load(argv[1], 0, &g) != SME_OK) { printf("load failed: %s\n", sme_last_error()); return 1; }
  sme_graph_info(g, &n, &m, &d);
  printf("n=%llu m=%llu dmax=%llu\n", (unsigned long long)n, (unsigned long long)m, (unsigned long long)d);
  sme_opts o;
  sme_opts_default(&o);
  printf("algo=%d mode=%d level=%d ordering=%d\n", o.algo, o.execute_mode, o.compress_level, o.enable_ordering);
  printf("q7_vertices=%d\n", sme_query_vertex_count(7));
  uint64_t need = 0;
  if (sme_plan_describe(3, 4, NULL, 0, &need) != SME_ERR_CAPACITY || need == 0) return 2;
  char* buf = (char*)malloc(need);
  if (sme_plan_describe(3, 4, buf, need, NULL) != SME_OK) return 3;
  printf("plan_bytes=%llu\n", (unsigned long long)need);
  free(buf);
  sme_graph* o2 = NULL;
  uint32_t* map = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  if (sme_graph_degree_order(g, 1, &o2, map) != SME_OK) return 4;
  printf("oriented=%d\n", sme_graph_is_oriented(o2));
  o.query_type = 1;
  uint64_t c = 0;
  sme_status st = sme_count(o2, &o, &c);
  printf("count_on_oriented_status=%d\n", (int)st);
  sme_graph_free(o2);
  free(map);
  o.query_type = 14;
  st = sme_count(g, &o, &c);
  printf("bad_query_status=%d\n", (int)st);
  sme_graph_free(g);
  printf("version=%s\n", sme_version());
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_plain_c_caller(tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(C_SRC)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "subgraphmatchgpu_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", libdir, "-lsme", f"-Wl,-rpath,{libdir}"], check=True)
    r = subprocess.run([str(exe), golden_graph_path("k12")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    assert "n=12 m=132 dmax=11" in out
    assert "algo=6 mode=1 level=3 ordering=1" in out
    assert "q7_vertices=5" in out
    assert "oriented=1" in out
    # 4-cycle on an oriented graph: refused at plan time (6), before any device work
    assert "count_on_oriented_status=6" in out
    assert "bad_query_status=6" in out
    assert "sm_100a" in out
