"""Generates the golden fixtures of the parity tests (run in a container that
has the reference sources; the outputs are committed).

* graphs/*.bin   small seeded graphs written by libsme's BIN writer
* counts.json    per (graph, query) the count printed by the reference's own
                 CPU program `patternmatchcpu -a 0` (CPU_WCOJ), built from the
                 reference sources by oracle/Makefile into oracle/_ref/
* plans/*.txt    the reference's own `test_plan` output (LIGHT plan with
                 NON_MATERIALIZE_OPT, reuse plan with autogen) per query
* preprocess.json  SHA-256 of the BIN file the reference's `preprocess_graph`
                 writes for a messy SNAP edge list, and of libsme's result for
                 the same text (they must be identical)

Usage:  python tests/golden/make_golden.py   (after `make -C oracle ref`)
"""
import hashlib
import json
import os
import random
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
import subgraphmatchgpu_b200 as sme  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

# name -> constructor; sizes keep every reference run within seconds
GRAPHS = {
    "k6": lambda: sme.Graph.clique(6),
    "k12": lambda: sme.Graph.clique(12),
    # the reference's own K20 cross-check graph (TestPatternMatchCPU.cpp:97-147)
    "k20": lambda: sme.Graph.clique(20),
    "rmat_s8_ef8": lambda: sme.Graph.rmat(8, 8, seed=11),
    "rmat_s10_ef8": lambda: sme.Graph.rmat(10, 8, seed=12),
    "rmat_s12_ef8": lambda: sme.Graph.rmat(12, 8, seed=13),
    "er_n600_d8": lambda: sme.Graph.er(600, 8.0, seed=14),
    "ba_n600_m4": lambda: sme.Graph.ba(600, 4, seed=15),
    "er_n64_d12": lambda: sme.Graph.er(64, 12.0, seed=16),
}
# queries too expensive for the reference on the larger graphs are skipped
SKIP = {
    ("rmat_s12_ef8", 5), ("rmat_s12_ef8", 9), ("rmat_s12_ef8", 10), ("rmat_s12_ef8", 13),
}


def ref_count(path: str, q: int) -> int:
    out = subprocess.run([os.path.join(REF, "patternmatchcpu"), "-f", path, "-d", "0", "-a", "0", "-q",
                          str(q), "-t", "8", "-b", "1"], capture_output=True, text=True, check=True).stdout
    m = re.search(r"total_match_count=(\d+)", out)
    return int(m.group(1))


def sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main():
    os.makedirs(os.path.join(HERE, "graphs"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "plans"), exist_ok=True)
    counts = {}
    for name, make in GRAPHS.items():
        g = make()
        path = os.path.join(HERE, "graphs", name + ".bin")
        g.write_bin(path)
        n, m, d = g.info()
        counts[name] = {"n": n, "m": m, "max_degree": d, "sha256": sha(path), "counts": {}}
        for q in range(14):
            if (name, q) in SKIP:
                continue
            counts[name]["counts"][str(q)] = ref_count(path, q)
        print(name, n, m, counts[name]["counts"], flush=True)
    with open(os.path.join(HERE, "counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)

    for q in range(14):
        for t, tag in ((1, "reuse_autogen"), (2, "light_nonmat_opt")):
            out = subprocess.run([os.path.join(REF, "test_plan"), "-a", "0", "-t", str(t), "-q", str(q)],
                                 capture_output=True, text=True, check=True).stdout
            with open(os.path.join(HERE, "plans", f"q{q}_{tag}.txt"), "w") as f:
                f.write(out)

    # preprocess byte-identity on a messy edge list (duplicates, both
    # directions, self loops, id gaps, a non-zero minimum id)
    rnd = random.Random(7)
    lines = ["# messy SNAP edge list"]
    for _ in range(3000):
        u, v = rnd.randrange(5, 400), rnd.randrange(5, 400)
        if rnd.random() < 0.3:
            v = u + rnd.randrange(0, 3)
        lines.append(f"{u}\t{v}")
        if rnd.random() < 0.2:
            lines.append(f"{v} {u}")
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "messy.txt")
        with open(txt, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([os.path.join(REF, "preprocess_graph"), "-f", txt, "-d", "0", "-o", "1"],
                       capture_output=True, check=True)
        ref_sha = sha(txt + ".bin")
        g = sme.Graph.load(txt, 0)
        g.preprocess()
        mine = os.path.join(td, "mine.bin")
        g.write_bin(mine)
        with open(os.path.join(HERE, "messy_edges.txt"), "w") as f:
            f.write("\n".join(lines) + "\n")
        res = {"reference_sha256": ref_sha, "libsme_sha256": sha(mine)}
    with open(os.path.join(HERE, "preprocess.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("preprocess", res)


if __name__ == "__main__":
    main()
