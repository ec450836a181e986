"""Generates the golden fixtures of the parity tests (run in a container that
has the reference sources; the outputs are committed).

* graphs/*.bin   small seeded graphs written by libsme's BIN writer
* counts.json    per (graph, query) the count printed by the reference's own
                 CPU program `patternmatchcpu -a 0` (CPU_WCOJ), built from the
                 reference sources by oracle/Makefile into oracle/_ref/
* plans/*.txt    the reference's own `test_plan` output (LIGHT plan with
                 NON_MATERIALIZE_OPT, reuse plan with autogen) per query, and
                 (q*_reuse_hardcoded.txt) the hard-coded reuse plan that
                 `patternmatchgpu -a 5` runs, printed with its vertex mappings
                 by oracle/_ref/ref_reuse_plan
* preprocess.json  SHA-256 of the BIN file the reference's `preprocess_graph`
                 writes for a messy SNAP edge list, and of libsme's result for
                 the same text (they must be identical)
* formats.json   SHA-256 of what the reference's `preprocess_graph` writes
                 as SNAP text (-o 0) and as ADJ text + info (-o 3) for that
                 edge list, and as BIN for an edge list with large, zero-padded
                 vertex names read through its .lvid reader (messy.lvid)

Usage:  python tests/golden/make_golden.py [formats|hardcoded]   (after
        `make -C oracle ref`; `formats` regenerates formats.json and messy.lvid
        only, `hardcoded` the hard-coded reuse plans only)
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


def formats():
    """The other graph formats of GraphIO, pinned against preprocess_graph."""
    res = {}
    messy = os.path.join(HERE, "messy_edges.txt")
    rnd = random.Random(9)
    names = [str(rnd.randrange(10 ** 9, 10 ** 14)) for _ in range(150)] + ["7", "007", "0", "00"]
    lines = ["# vertex names beyond 32 bits, zero-padded duplicates of small ids"]
    for _ in range(1200):
        u, v = rnd.choice(names), rnd.choice(names)
        sep = rnd.choice(["\t", " ", ", ", " ; "])
        lines.append(f"{u}{sep}{v}")
    lvid = os.path.join(HERE, "messy.lvid")
    with open(lvid, "w") as f:
        f.write("\n".join(lines) + "\n")
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "messy.txt")
        with open(messy) as src, open(txt, "w") as dst:
            dst.write(src.read())
        for fmt, suffix in ((0, ".snap.txt"), (3, ".adj.txt")):
            subprocess.run([os.path.join(REF, "preprocess_graph"), "-f", txt, "-d", "0", "-o", str(fmt)],
                           capture_output=True, check=True)
            res[f"reference{suffix}"] = sha(txt + suffix)
        with open(txt + ".adj.txt.info") as f:
            res["reference.adj.txt.info"] = f.read()
        g = sme.Graph.load(txt, 0)
        g.preprocess()
        g.write_snap(os.path.join(td, "mine.snap"))
        g.write_adj(os.path.join(td, "mine.adj"))
        res["libsme.snap.txt"] = sha(os.path.join(td, "mine.snap"))
        res["libsme.adj.txt"] = sha(os.path.join(td, "mine.adj"))
        with open(os.path.join(td, "mine.adj.info")) as f:
            res["libsme.adj.txt.info"] = f.read()
        tl = os.path.join(td, "messy.lvid")
        with open(lvid) as src, open(tl, "w") as dst:
            dst.write(src.read())
        subprocess.run([os.path.join(REF, "preprocess_graph"), "-f", tl, "-d", "0", "-o", "1"],
                       capture_output=True, check=True)
        res["reference.lvid.bin"] = sha(tl + ".bin")
        g = sme.Graph.load(tl, 0)
        g.preprocess()
        g.write_bin(os.path.join(td, "mine_lvid.bin"))
        res["libsme.lvid.bin"] = sha(os.path.join(td, "mine_lvid.bin"))
    with open(os.path.join(HERE, "formats.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print("formats", res)


# queries with a hard-coded reuse plan (Q1 and Q4 end in the reference's assert)
HARDCODED = (0, 2, 3, 5, 6, 7, 8, 9, 10, 11, 12, 13)


def hardcoded():
    os.makedirs(os.path.join(HERE, "plans"), exist_ok=True)
    for q in HARDCODED:
        out = subprocess.run([os.path.join(REF, "ref_reuse_plan"), str(q)], capture_output=True, text=True,
                             check=True).stdout
        with open(os.path.join(HERE, "plans", f"q{q}_reuse_hardcoded.txt"), "w") as f:
            f.write(out)


if __name__ == "__main__":
    if sys.argv[1:] == ["formats"]:
        formats()
    elif sys.argv[1:] == ["hardcoded"]:
        hardcoded()
    else:
        main()
        formats()
        hardcoded()
