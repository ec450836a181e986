#!/usr/bin/env python3
"""Benchmark of the GPU subgraph-enumeration path (one JSON line on rank 0).

Workload: the 4-clique (Q3), 4-cycle (Q1) and diamond (Q2) counts, with the
reference's symmetry-breaking constraints, on an undirected R-MAT graph of
scale 20, edge factor 16, a/b/c/d = .57/.19/.19/.05, seed 20, generated here
with numpy and passed through the reference's preprocessing (self loops and
parallel edges dropped, dangling vertices dropped with an order-preserving
relabel), uint32 CSR, uint64 counts.

A step is one query over one root task: a block of roots drawn from a seeded
permutation of the vertices of degree <= 1024 (99% of the roots).  Both arms
run the same steps in the same order:

  * this engine (default arm): sme_count with the LIGHT plan on the resident
    graph; `value` = instances / CUDA-event device time; `e2e` = the same
    steps through sme_count with the CSR in pinned host memory copied to the
    device in every step;
  * the reference (`--impl reference`): the reference's own CPU_WCOJ DFS over
    the same root blocks (oracle/_ref/ref_wcoj_task, compiled from its
    sources) on the BIN file its own preprocess_graph wrote from the same edge
    list, with every host thread.

Hub roots (degree > 1024) are left out of the shared steps because the
reference's per-root DFS cannot finish one in bounded time (a single hub root
of the 4-clique runs for minutes on eight cores).  The engine's whole-graph
counts, hubs included, are reported in `whole_graph`.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sme|reference]
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "instances/sec (4-clique, 4-cycle, diamond; R-MAT s20 ef16)"
UNIT = "instances/s"
QUERY_NAMES = {0: "triangle", 1: "4-cycle", 2: "diamond", 3: "4-clique", 4: "house", 7: "5-clique"}
REF_TASK = os.path.join(ROOT, "oracle", "_ref", "ref_wcoj_task")
REF_PREPROCESS = os.path.join(ROOT, "oracle", "_ref", "preprocess_graph")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sme", choices=["sme", "reference"])
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=20)
    ap.add_argument("--queries", default="3,1,2")
    ap.add_argument("--algo", type=int, default=6)
    ap.add_argument("--hub-degree", type=int, default=1024, help="roots above this degree are not in the shared steps")
    ap.add_argument("--blocks", default="3:16384,1:512,2:8192", help="roots per step, per query")
    ap.add_argument("--check-algo", type=int, default=4, help="second plan that recounts every timed step")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched / served measurements")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--task-roots", type=int, default=256, help="served: roots per request task")
    ap.add_argument("--rates", default="50,500,5000", help="served: open-loop arrival rates (req/s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--granularity", type=int, default=0,
                    help="0 auto (specialised warp per path), 1 warp per path generic, 2 flattened, "
                         "3 specialised at six blocks per SM")
    ap.add_argument("--list-only", action="store_true", help="no hub bitmaps (comparison)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-pack", action="store_true", help="end to end with the plain uint32 CSR upload only")
    ap.add_argument("--no-whole", action="store_true", help="skip the whole-graph counts")
    ap.add_argument("--no-s22", action="store_true", help="skip the R-MAT s22 legs")
    ap.add_argument("--no-l2-flush", action="store_true", help="do not flush L2 between steps")
    ap.add_argument("--threads", type=int, default=0, help="CPU threads (0: all)")
    ap.add_argument("--profile-house", type=int, default=0,
                    help="N: only count the house (LIGHT) on the bench graph over the first N roots of degree "
                         "<= hub_degree in a seeded order once (a small case for a profiler capture) and exit")
    ap.add_argument("--profile-upload", type=int, default=0,
                    help="N: only run N counts of the first diamond step on the bench graph held packed in host "
                         "memory (every call uploads and expands it; a small case for a profiler capture) and exit")
    ap.add_argument("--profile-s22", default="",
                    help="BEGIN:END:STRIDE: only count the 4-clique of the degree-oriented R-MAT s22 graph over "
                         "roots BEGIN, BEGIN+STRIDE, ... < END once (a small case for a profiler capture), print "
                         "its stats and exit")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- workload --
def rmat_edges(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=20):
    """R-MAT edge list: n * edge_factor edges, each picking one quadrant per
    level (a top-left, b top-right, c bottom-left, d bottom-right) from one
    uniform draw; vertex ids are the concatenated bits (no relabelling)."""
    rng = np.random.default_rng(seed)
    ne = (1 << scale) * edge_factor
    u = np.zeros(ne, np.uint32)
    v = np.zeros(ne, np.uint32)
    ab, abc = a + b, a + b + c
    one = np.uint32(1)
    for _ in range(scale):
        r = rng.random(ne)
        u = (u << one) | (r >= ab).astype(np.uint32)
        v = (v << one) | (((r >= a) & (r < ab)) | (r >= abc)).astype(np.uint32)
    return u, v


def raw_csr(u, v, n):
    """Undirected CSR of an edge list as the reference's SNAP reader builds it
    (both directions, lists sorted, self loops and parallel edges kept): the
    input of the preprocessing step."""
    keys = np.concatenate([(u.astype(np.uint64) << np.uint64(32)) | v, (v.astype(np.uint64) << np.uint64(32)) | u])
    keys.sort()
    src = (keys >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.uint64)
    rp[1:] = np.cumsum(np.bincount(src, minlength=n), dtype=np.uint64)
    return rp, (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def csr_digest(rp, cl):
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(rp, np.uint64).tobytes())
    h.update(np.ascontiguousarray(cl, np.uint32).tobytes())
    return h.hexdigest()[:16]


def parse_blocks(spec):
    return {int(k): int(v) for k, v in (x.split(":") for x in spec.split(","))}


def make_steps(rp, args, count):
    """The first `count` steps: step i is query qs[i % len(qs)] over block
    i // len(qs) of that query's seeded permutation of the roots of degree
    <= hub_degree (blocks wrap around the permutation)."""
    qs = [int(q) for q in args.queries.split(",")]
    blocks = parse_blocks(args.blocks)
    deg = np.diff(np.asarray(rp, np.uint64)).astype(np.int64)
    pool = np.flatnonzero(deg <= args.hub_degree).astype(np.uint32)
    perms = {q: np.random.default_rng(args.seed * 1000 + q).permutation(pool) for q in qs}
    steps = []
    for i in range(count):
        q = qs[i % len(qs)]
        k = i // len(qs)
        p, bsz = perms[q], min(blocks[q], len(pool))
        start = (k * bsz) % max(len(p), 1)
        idx = (start + np.arange(bsz)) % max(len(p), 1)
        steps.append((q, np.ascontiguousarray(p[idx], np.uint32)))
    return steps


def config_of(args, n, m, digest):
    blocks = parse_blocks(args.blocks)
    qs = [int(q) for q in args.queries.split(",")]
    return {"workload": f"R-MAT s{args.scale} ef{args.edge_factor} (a,b,c)=(.57,.19,.19) seed {args.seed}, numpy "
                        f"generator + the reference's preprocessing: n={n} m={m} csr_sha1={digest}; queries "
                        + ", ".join(f"Q{q} {QUERY_NAMES.get(q, q)}" for q in qs) +
                        " with the reference's symmetry breaking; a step = one query over one block of roots "
                        f"drawn from a seeded permutation of the roots of degree <= {args.hub_degree} (roots "
                        "per block: " + ", ".join(f"Q{q} {blocks[q]}" for q in qs) + ")",
            "plan": f"algo {args.algo} (6 = LIGHT), IN_MEMORY_GPU",
            "l2": "GPU arm: L2 flushed before every step (256 MiB write, outside the timed region); "
                  "inputs: CSR %d bytes" % (8 * (n + 1) + 4 * m),
            "parallelism": "single GPU (replicas when N > 1)"}


def per_query_summary(per_q):
    return {str(q): {"name": QUERY_NAMES.get(q, str(q)), "instances": int(v[0]), "seconds": v[1],
                     "value": (v[0] / v[1]) if v[1] > 0 else 0.0, "steps": v[2]} for q, v in sorted(per_q.items())}


# ----------------------------------------------------------- measurement --
class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    polled every 5 ms from a thread (the timed steps take tens of ms, too short
    for nvidia-smi's sampling loop); the device is found by its PCI bus id, so
    the index a process sees under CUDA_VISIBLE_DEVICES does not matter.
    nvidia-smi at 200 ms is the fallback."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []
        self.h = None
        self.stop_flag = False

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.h = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def _poll(self):
        nv = self.nv
        mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        while not self.stop_flag:
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM), mx,
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(self.h), time.perf_counter()))
            except Exception:
                break
            time.sleep(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        if self.h is not None:
            self.stop_flag = True
            self.t.join(timeout=5)
            nv = self.nv
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
            timed = [x for x in self.samples if t0 <= x[3] <= t1]
            use, window = (timed, "timed steps") if len(timed) >= 3 else (self.samples, "warm-up and timed steps")
            reasons = {n for _, _, r, _ in use for n, b in zip(names, bits) if r & b}
            sm = [c for c, _, _, _ in use]
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": self.samples[0][1] if self.samples else None,
                    "reasons": sorted(reasons), "samples": len(sm), "timed_samples": len(timed),
                    "window": window, "source": "NVML, 5 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def reduce_over_ranks(dev_ms, instances, dist, device):
    """Replicas: the job's time is the slowest rank's device time, its work
    the sum of the ranks' instances (timing only; no data-path collective)."""
    if dist is None:
        return dev_ms, float(instances)
    import torch
    tmax = torch.tensor([float(dev_ms)], dtype=torch.float64, device=device)
    tsum = torch.tensor([float(instances)], dtype=torch.float64, device=device)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax.item()), float(tsum.item())


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# ------------------------------------------------------ the reference's CPU --
def threads_of(args):
    return args.threads or os.cpu_count() or 1


def reference_tasks(bin_path, steps, threads, tmpdir):
    """Runs the reference's CPU_WCOJ over each step's roots with the task
    driver built from its sources; returns [(count, elapsed_ms)] per step.
    One driver process per query (the graph loads once per query)."""
    out = [None] * len(steps)
    for q in sorted({s[0] for s in steps}):
        idx = [i for i, s in enumerate(steps) if s[0] == q]
        roots = np.concatenate([steps[i][1] for i in idx]) if idx else np.zeros(0, np.uint32)
        rpath = os.path.join(tmpdir, f"roots_q{q}.u32")
        roots.astype(np.uint32).tofile(rpath)
        args, off = [], 0
        for i in idx:
            args.append(f"L:{off}:{len(steps[i][1])}")
            off += len(steps[i][1])
        r = subprocess.run([REF_TASK, "-f", bin_path, "-q", str(q), "-t", str(threads), "-r", rpath] + args,
                           capture_output=True, text=True, check=True)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("task=")]
        if len(lines) != len(idx):
            raise RuntimeError(f"reference task driver printed {len(lines)} results for {len(idx)} tasks")
        for i, ln in zip(idx, lines):
            kv = dict(x.strip().split("=", 1) for x in ln.split(","))
            out[i] = (int(kv["total_match_count"]), float(kv["elapsed_time"].rstrip("ms")))
    return out


def port_tasks(rp, cl, steps, threads):
    """The oracle's C restatement of CPU_WCOJ over the same steps (used when
    the reference's own driver was not built)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as O
    out = []
    for q, roots in steps:
        t0 = time.perf_counter()
        c = O.count_roots(rp, cl, q, roots, threads)
        out.append((c, (time.perf_counter() - t0) * 1e3))
    return out


def reference_graph(args, tmpdir):
    """The edge list through the reference's own preprocess_graph into its BIN
    file; (bin path, row_ptrs, cols).  Without the reference's tools the
    oracle's numpy restatement of the same preprocessing is used and the BIN
    path is None."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as O
    u, v = rmat_edges(args.scale, args.edge_factor, seed=args.seed)
    if os.path.exists(REF_PREPROCESS) and os.path.exists(REF_TASK):
        txt = os.path.join(tmpdir, "rmat.txt")
        O.write_edge_text(u, v, txt)
        subprocess.run([REF_PREPROCESS, "-f", txt, "-d", "0"], capture_output=True, text=True, check=True)
        rp, cl = O.read_bin(txt + ".bin")
        return txt + ".bin", rp, cl
    rp, cl = raw_csr(u, v, 1 << args.scale)
    return None, *O.preprocess_csr(rp, cl)


def calibrate_c1(threads, tmp):
    """The reference's unmodified CPU program (patternmatchcpu -a 0 -q 0) on
    the triangle configuration (R-MAT s14 ef8, the reference's own
    elapsed_time=, src/cpu/PatternMatchCPU.cpp:55-62 and CPUWCOJ.h:58-60),
    beside the root-task driver over all roots of the same BIN: the driver
    runs the same DFS, so their times should agree."""
    binary = os.path.join(ROOT, "oracle", "_ref", "patternmatchcpu")
    if not (os.path.exists(binary) and os.path.exists(REF_TASK) and os.path.exists(REF_PREPROCESS)):
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as O
    u, v = rmat_edges(14, 8, seed=14)
    txt = os.path.join(tmp, "c1.txt")
    O.write_edge_text(u, v, txt)
    subprocess.run([REF_PREPROCESS, "-f", txt, "-d", "0"], capture_output=True, text=True, check=True)
    out = subprocess.run([binary, "-f", txt + ".bin", "-d", "0", "-a", "0", "-q", "0", "-t", str(threads)],
                         capture_output=True, text=True, check=True).stdout
    line = next(ln for ln in out.splitlines() if ln.startswith("total_match_count="))
    kv = dict(x.strip().split("=", 1) for x in line.split(","))
    c, ms = int(kv["total_match_count"]), float(kv["elapsed_time"].rstrip("ms"))
    drv = subprocess.run([REF_TASK, "-f", txt + ".bin", "-q", "0", "-t", str(threads), "S:1:0"],
                         capture_output=True, text=True, check=True).stdout
    dk = dict(x.strip().split("=", 1) for x in next(ln for ln in drv.splitlines() if ln.startswith("task=")).split(","))
    return {"workload": "R-MAT s14 ef8 seed 14, triangle, whole graph", "threads": threads,
            "patternmatchcpu": {"instances": c, "elapsed_ms": ms, "value": c / (ms / 1e3) if ms > 0 else 0.0},
            "ref_wcoj_task": {"instances": int(dk["total_match_count"]),
                              "elapsed_ms": float(dk["elapsed_time"].rstrip("ms"))}}


def run_reference(args, rank, world):
    """CPU reference arm: the reference's own CPU_WCOJ on the host cores, the
    same steps as the engine's arm (rank 0 only; other ranks exit)."""
    if rank != 0:
        return
    threads = threads_of(args)
    with tempfile.TemporaryDirectory() as tmp:
        bin_path, rp, cl = reference_graph(args, tmp)
        n, m = len(rp) - 1, len(cl)
        steps = make_steps(rp, args, args.warmup + args.steps)
        if bin_path:
            res = reference_tasks(bin_path, steps, threads, tmp)
            kind, what = "reference", ("the reference's CPU_WCOJ DFS (src/cpu/CPUWCOJ.h) compiled from its sources "
                                       "(oracle/_ref/ref_wcoj_task) on the BIN its preprocess_graph wrote")
        else:
            res = port_tasks(rp, cl, steps, threads)
            kind, what = "port", "the oracle's C restatement of CPU_WCOJ (the reference's tools were not built)"
        try:
            c1 = calibrate_c1(threads, tmp)
        except Exception as ex:  # reported in the line, never dropped silently
            c1 = {"error": f"{type(ex).__name__}: {ex}"}
    timed = list(zip(steps, res))[args.warmup:]
    inst = sum(c for _, (c, _) in timed)
    ms = sum(t for _, (_, t) in timed)
    per_q = {}
    for (q, roots), (c, t) in timed:
        e = per_q.setdefault(q, [0, 0.0, 0])
        e[0] += c
        e[1] += t / 1e3
        e[2] += 1
    value = inst / (ms / 1e3) if ms > 0 else 0.0
    cb = {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
          "sample": f"{what}; the {args.steps} timed steps of the shared step list, {threads} OpenMP threads; "
                    f"{inst} instances in {ms / 1e3:.2f} s"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": config_of(args, n, m, csr_digest(rp, cl)), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "per_query": per_query_summary(per_q),
            "step_counts": [int(c) for _, (c, _) in timed], "c1_calibration": c1}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- engine --
def engine_graph(args):
    """The same edge list through the engine's preprocessing
    (sme_graph_preprocess, the reference's PreprocessGraph semantics)."""
    import subgraphmatchgpu_b200 as sme
    u, v = rmat_edges(args.scale, args.edge_factor, seed=args.seed)
    rp, cl = raw_csr(u, v, 1 << args.scale)
    g = sme.Graph.from_csr(rp, cl)
    g.preprocess()
    g.validate()
    return g


def cpu_baseline(args, g, steps, gpu_counts):
    """The reference's CPU_WCOJ (or the oracle port) on the host cores over the
    first timed step of each query: its rate, and its counts against the
    engine's counts of the same steps."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    threads = threads_of(args)
    first = {}
    for i, (q, _) in enumerate(steps):
        first.setdefault(q, i)
    pick = sorted(first.values())
    sub = [steps[i] for i in pick]
    with tempfile.TemporaryDirectory() as tmp:
        if os.path.exists(REF_TASK):
            path = os.path.join(tmp, "g.bin")
            g.write_bin(path)
            res = reference_tasks(path, sub, threads, tmp)
            kind = "reference"
        else:
            rp, cl = g.csr()
            res = port_tasks(rp, cl, sub, threads)
            kind = "port"
    inst = sum(c for c, _ in res)
    ms = sum(t for _, t in res)
    per_q = {q: [c, t / 1e3, 1] for (q, _), (c, t) in zip(sub, res)}
    return {"value": inst / (ms / 1e3) if ms > 0 else 0.0, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{'the reference CPU_WCOJ task driver' if kind == 'reference' else 'oracle port'} over the "
                      f"first timed step of each query ({len(sub)} steps), {threads} threads",
            "per_query": per_query_summary(per_q),
            "counts_equal_gpu": all(int(c) == int(gpu_counts[i]) for i, (c, _) in zip(pick, res))}


def small_graph_batch(num, seed):
    """The batched configuration: graphs log-uniform over 64..4096 vertices,
    half Erdos-Renyi and half Barabasi-Albert, average degree U[4, 32];
    queries uniform over triangle, 4-cycle, diamond, 4-clique."""
    import random
    import subgraphmatchgpu_b200 as sme
    rnd = random.Random(seed)
    gs, qs = [], []
    for i in range(num):
        n = int(round(2 ** rnd.uniform(6, 12)))
        d = rnd.uniform(4, 32)
        if i % 2 == 0:
            gs.append(sme.Graph.er(n, d, seed=seed * 100003 + i))
        else:
            gs.append(sme.Graph.ba(n, max(1, int(round(d / 2))), seed=seed * 100003 + i))
        qs.append(rnd.choice([0, 1, 2, 3]))
    return gs, qs


def bench_batched(args, device):
    """Batched form vs the plain path (one sme_count per graph, graph copied
    to the device per call) on the same small graphs; every graph's count is
    checked against the CPU oracle."""
    import subgraphmatchgpu_b200 as sme
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as O
    gs, qs = small_graph_batch(args.batch_graphs, 77)
    t0 = time.perf_counter()
    plan = sme.BatchPlan(gs, qs, autotune=True, use_graph=True, device=device)
    prep_s = time.perf_counter() - t0
    counts, _ = plan.run()
    runs = []
    for _ in range(3):
        c, t = plan.run()
        runs.append(t)
        if not np.array_equal(c, counts):
            raise RuntimeError("batched counts differ between replays")
    ms = min(runs)
    total = int(counts.sum())
    t0 = time.perf_counter()
    plain = [g.count(q, sme.GPU_LIGHT, device=device) for g, q in zip(gs, qs)]
    plain_s = time.perf_counter() - t0
    ok_plain = all(int(a) == int(b) for a, b in zip(plain, counts))
    # every graph against the CPU oracle, graphs spread over the host threads
    # (the oracle's ctypes calls release the GIL)
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    csrs = [g.csr() for g in gs]
    with ThreadPoolExecutor(max_workers=threads_of(args)) as ex:
        cpu = list(ex.map(lambda i: O.count(*csrs[i], qs[i], threads=1), range(len(gs))))
    bad = [i for i in range(len(gs)) if cpu[i] != int(counts[i])]
    cpu_s = time.perf_counter() - t0
    d = plan.describe()
    plan.close()
    return {"graphs": len(gs), "instances": total,
            "batched": {"value": total / (ms / 1e3), "unit": UNIT, "ms": ms, "prepare_autotune_s": prep_s,
                        "group_threads": d["group_threads"], "block_threads": d["block_threads"],
                        "items_per_fetch": d["items_per_fetch"], "tuned_ms": d["tuned_ms"],
                        "work_items": d["work_items"], "cuda_graph": True,
                        "tuner": "group of 4/8/16 lanes, a warp, or 64/128 threads of a CTA per item x block "
                                 "128/256/512, then 1/4/16 items per fetch"},
            "plain": {"value": total / plain_s, "unit": UNIT, "ms": plain_s * 1e3},
            "counts_equal_plain": ok_plain, "counts_equal_cpu": not bad, "cpu_checked_graphs": len(gs),
            "cpu_mismatches": bad[:8], "cpu_check_s": round(cpu_s, 2)}


def bench_served(args, device):
    """Served form: each request is one pattern on a root task of a resident
    R-MAT graph (s16/s18/s20, ef16) or on an attached Erdos-Renyi graph
    (256..8192 vertices, degree 8).  Closed loop (everything queued) and open
    loops with Poisson arrivals at each rate, against the same requests run
    one at a time through the plain path in arrival order."""
    import random
    import subgraphmatchgpu_b200 as sme
    rnd = random.Random(5)
    resident = [sme.Graph.rmat(s, 16, seed=100 + s) for s in (16, 18, 20)]
    for g in resident:
        g.to_device(device)
    srv = sme.Server(slots=args.slots, device=device)
    gids = [srv.add_graph(g) for g in resident]
    pats = [0, 1, 2, 3, 4, 7]
    reqs = []
    for i in range(args.requests):
        q = rnd.choice(pats)
        if rnd.random() < 0.5:
            n = rnd.randint(256, 8192)
            reqs.append((q, -1, sme.Graph.er(n, 8.0, seed=9000 + i), 0, 0, 1))
        else:
            k = rnd.randrange(3)
            n = resident[k].n
            stride = max(1, n // args.task_roots)
            reqs.append((q, gids[k], None, rnd.randrange(stride), n, stride))

    def plain_run(r):
        q, gid, att, a, b, st = r
        g = att if att is not None else resident[gid]
        return g.count(q, sme.GPU_LIGHT, root_begin=a, root_end=b, root_stride=st, device=device)

    def submit(r):
        q, gid, att, a, b, st = r
        return srv.submit(q, gid=gid, attached=att, root_begin=a, root_end=b, root_stride=st)

    t0 = time.perf_counter()
    plain_counts = [plain_run(r) for r in reqs]
    plain_s = time.perf_counter() - t0
    inst = int(sum(plain_counts))
    t0 = time.perf_counter()
    ids = [submit(r) for r in reqs]
    closed = [srv.wait(i) for i in ids]
    served_s = time.perf_counter() - t0
    same = [x[0] for x in closed] == plain_counts

    def arrivals(rate, seed):
        gen = random.Random(seed)
        t = time.perf_counter()
        for _ in reqs:
            t += gen.expovariate(rate)
            yield t

    open_loop = []
    for rate in [float(x) for x in args.rates.split(",")]:
        lat_plain, t_busy = [], time.perf_counter()
        for r, t_arr in zip(reqs, arrivals(rate, int(rate))):
            while time.perf_counter() < t_arr:
                time.sleep(0.0002)
            plain_run(r)
            lat_plain.append((time.perf_counter() - t_arr) * 1e3)
        plain_wall = time.perf_counter() - t_busy
        ids, t_busy = [], time.perf_counter()
        for r, t_arr in zip(reqs, arrivals(rate, int(rate))):
            while time.perf_counter() < t_arr:
                time.sleep(0.0002)
            ids.append(submit(r))
        got = [srv.wait(i) for i in ids]
        served_wall = time.perf_counter() - t_busy
        same = same and [x[0] for x in got] == plain_counts
        lat = [x[1] for x in got]
        open_loop.append({"arrival_rate_per_s": rate,
                          "served": {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                     "value": inst / served_wall, "unit": UNIT},
                          "plain": {"p50_ms": float(np.percentile(lat_plain, 50)),
                                    "p99_ms": float(np.percentile(lat_plain, 99)),
                                    "value": inst / plain_wall, "unit": UNIT}})
    stats = srv.stats()
    srv.close()
    return {"requests": len(reqs), "slots": args.slots, "instances": inst,
            "closed_loop": {"served": {"value": inst / served_s, "unit": UNIT, "s": served_s},
                            "plain": {"value": inst / plain_s, "unit": UNIT, "s": plain_s}},
            "open_loop": open_loop, "max_inflight": stats["max_inflight"],
            "counts_equal_alone_and_in_mix": same}


def leg_roofline(s, peak):
    """Roofline of the intersection kernels of one run (sme_last_stats)."""
    ach = s.algorithmic_bytes / (s.kernel_ms / 1e3) / 1e9 if s.kernel_ms > 0 else 0.0
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "kernel_ms": round(s.kernel_ms, 3), "algorithmic_bytes": int(s.algorithmic_bytes),
            "launches": int(s.hot_launches)}


def bench_whole_graph(args, g, device, tune, peak):
    """The engine alone on the whole configuration, hubs included: 4-clique
    and diamond over every root, the 4-cycle over every 64th root (its full
    count takes minutes); each count checked against the reuse plan."""
    import subgraphmatchgpu_b200 as sme
    out = {}
    for q, stride in ((3, 1), (2, 1), (1, 64)):
        c = g.count(q, args.algo, root_stride=stride, device=device, **tune)
        s = sme.last_stats()
        check = g.count(q, sme.GPU_GPSM_REUSE, root_stride=stride, device=device, **tune)
        out[str(q)] = {"name": QUERY_NAMES[q], "roots": "all" if stride == 1 else f"every {stride}th",
                       "instances": c, "device_ms": s.device_ms, "value": c / (s.device_ms / 1e3), "unit": UNIT,
                       "roofline": leg_roofline(s, peak), "count_equals_reuse_plan": c == check}
    inst = sum(v["instances"] for v in out.values())
    ms = sum(v["device_ms"] for v in out.values())
    out["all"] = {"instances": inst, "device_ms": ms, "value": inst / (ms / 1e3), "unit": UNIT}
    return out


def bench_s22(args, device, tune, peak):
    """R-MAT scale 22, edge factor 16: the 4-clique on the degree-ordered
    orientation (whole graph), the 5-clique (LIGHT and reuse plans, every
    16th root, oriented), the house (LIGHT, a block of roots) and the
    external mode with a device budget below the CSR size.  Each leg reports
    its own error instead of ending the others."""
    import subgraphmatchgpu_b200 as sme
    g = sme.Graph.rmat(22, args.edge_factor, 0.57, 0.19, 0.19, seed=22)
    o, _ = g.degree_order(orient=True)
    n, m, _ = g.info()
    out = {"workload": f"R-MAT s22 ef{args.edge_factor} seed 22 (libsme generator; n={n}, m={m}); cliques on "
                       "the degree-ordered orientation"}

    def leg(name, fn):
        try:
            out[name] = fn()
        except Exception as ex:  # reported in the line, never dropped silently
            out[name] = {"error": f"{type(ex).__name__}: {ex}"}

    def run(gr, q, algo, **kw):
        c = gr.count(q, algo, device=device, **kw)
        s = sme.last_stats()
        return c, {"instances": c, "device_ms": s.device_ms, "value": c / (s.device_ms / 1e3), "unit": UNIT,
                   "roofline": leg_roofline(s, peak)}

    o.to_device(device)
    clique4 = {}

    def four():
        c, r = run(o, 3, args.algo, **tune)
        clique4["count"] = c
        c5, _ = run(o, 3, sme.GPU_GPSM_REUSE, **tune)
        r["count_equals_reuse_plan"] = c == c5
        return r

    def five():
        r5 = {"roots": "every 16th"}
        for algo in (sme.GPU_LIGHT, sme.GPU_GPSM_REUSE):
            _, r5[str(algo)] = run(o, 7, algo, root_stride=16, **tune)
        r5["counts_equal"] = r5["6"]["instances"] == r5["5"]["instances"]
        return r5

    leg("4clique_oriented", four)
    leg("5clique_oriented", five)
    o.release_device()

    def house():
        # the LIGHT house plan roots its tasks at pattern vertex u1 (search
        # sequence 1 2 3 0 4): the check is the same plan with every vertex
        # materialised (compress level 0)
        g.to_device(device)
        deg = np.diff(g.csr()[0]).astype(np.int64)
        roots = np.random.default_rng(22).permutation(np.flatnonzero(deg <= args.hub_degree))[:4096]
        roots = roots.astype(np.uint32)
        c, r = run(g, 4, sme.GPU_LIGHT, roots=roots, **tune)
        c0, _ = run(g, 4, sme.GPU_LIGHT, roots=roots, compress_level=0, **tune)
        g.release_device()
        r.update({"roots": f"4096 random roots of degree <= {args.hub_degree}",
                  "count_equals_compress_level_0": c == c0})
        return r

    def external():
        csr_bytes = 8 * (o.n + 1) + 4 * o.m
        budget = 256 << 20
        t0 = time.perf_counter()
        ce = o.count(3, sme.GPU_LIGHT, mode=sme.EXTERNAL_GPU, mem_limit_bytes=budget, device=device)
        wall = time.perf_counter() - t0
        s = sme.last_stats()
        return {"mem_limit_bytes": budget, "csr_bytes": csr_bytes, "instances": ce, "wall_s": wall,
                "device_ms": s.device_ms, "value": ce / wall, "unit": UNIT, "h2d_bytes": int(s.h2d_bytes),
                "batches": int(s.batches), "external_load_ms": s.phase_ms[7],
                "count_equals_in_memory": ce == clique4.get("count")}

    leg("house", house)
    leg("external_4clique_oriented", external)
    return out


def profile_house(args):
    """One count of the house (LIGHT plan) on the bench's R-MAT graph over a
    block of non-hub roots (the plan roots the house at u1), resident: the
    house's kernels for a profiler capture."""
    import subgraphmatchgpu_b200 as sme
    g = engine_graph(args)
    rp, _ = g.csr()
    deg = np.diff(rp).astype(np.int64)
    roots = np.random.default_rng(args.seed * 1000 + 4).permutation(np.flatnonzero(deg <= args.hub_degree))
    roots = roots[:args.profile_house].astype(np.uint32)
    g.to_device(0)
    c = g.count(4, sme.GPU_LIGHT, roots=roots, warp_granularity=args.granularity)
    s = sme.last_stats()
    print(json.dumps({"roots": len(roots), "instances": c, "device_ms": s.device_ms, "kernel_ms": s.kernel_ms,
                      "algorithmic_bytes": s.algorithmic_bytes, "launches": s.kernel_launches,
                      "hot_launches": s.hot_launches, "phase_ms": list(s.phase_ms)}), flush=True)


def profile_upload(args):
    """N counts of the first diamond step on the bench graph, not resident and
    held packed: each call copies the packed lists in ranges, expands them and
    builds the hub bitmaps before counting (the upload kernels for a profiler
    capture)."""
    import subgraphmatchgpu_b200 as sme
    g = engine_graph(args)
    rp, _ = g.csr()
    packed = g.pack()
    q, roots = next((q, r) for q, r in make_steps(rp, args, 3) if q == 2)
    out = []
    for _ in range(args.profile_upload):
        c = g.count(q, sme.GPU_LIGHT, roots=roots)
        s = sme.last_stats()
        out.append({"instances": c, "elapsed_ms": s.elapsed_ms, "device_ms": s.device_ms, "h2d_bytes": s.h2d_bytes})
    print(json.dumps({"packed_bytes": packed, "calls": out}), flush=True)


def bench_noalloc(device):
    """sme_count_noalloc beside sme_count on one resident R-MAT graph: the
    allocation-free path trades parallelism for its fixed scratch array."""
    import ctypes
    import subgraphmatchgpu_b200 as sme
    g = sme.Graph.rmat(16, 16, seed=16)
    g.to_device(device)
    d_rp, d_cl = g.device_arrays(device)
    out = {"graph": "R-MAT s16 ef16 seed 16 (library generator)", "n": g.n, "m": g.m,
           "max_degree": g.info()[2], "queries": {}}
    # the triangle only: on this graph the 4-clique takes the allocation-free
    # path about 10 s and the 4-cycle about 100 s (sme_count: 11 and 167 ms)
    for q in (0,):
        g.count(q, device=device)
        t0 = time.perf_counter()
        want = g.count(q, device=device)
        t_count = time.perf_counter() - t0
        got = ctypes.c_uint64()
        sme.lib().sme_count_noalloc(d_rp, d_cl, g.n, q, ctypes.byref(got))
        t0 = time.perf_counter()
        st = sme.lib().sme_count_noalloc(d_rp, d_cl, g.n, q, ctypes.byref(got))
        t_noalloc = time.perf_counter() - t0
        out["queries"][QUERY_NAMES.get(q, str(q))] = {
            "sme_count_ms": round(t_count * 1e3, 3), "sme_count_noalloc_ms": round(t_noalloc * 1e3, 3),
            "status": st, "counts_equal": st == 0 and got.value == want, "instances": want}
    g.release_device()
    return out


def profile_s22(args):
    """One count of the 4-clique over a root range of the degree-oriented
    R-MAT s22 ef16 graph (the graph of the s22 legs), resident, with the
    device footprint kept small: the case a profiler capture replays."""
    import subgraphmatchgpu_b200 as sme
    b, e, st = (int(x) for x in args.profile_s22.split(":"))
    g = sme.Graph.rmat(22, args.edge_factor, 0.57, 0.19, 0.19, seed=22)
    o, _ = g.degree_order(orient=True)
    del g
    o.to_device(0)
    c = o.count(3, args.algo, root_begin=b, root_end=e, root_stride=st, mem_limit_bytes=2 << 30,
                warp_granularity=args.granularity)
    s = sme.last_stats()
    print(json.dumps({"roots": [b, e, st], "instances": c, "device_ms": s.device_ms, "kernel_ms": s.kernel_ms,
                      "algorithmic_bytes": s.algorithmic_bytes, "launches": s.kernel_launches,
                      "hot_launches": s.hot_launches, "phase_ms": list(s.phase_ms)}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile_s22:
        return profile_s22(args)
    if args.profile_house:
        return profile_house(args)
    if args.profile_upload:
        return profile_upload(args)

    import torch
    import subgraphmatchgpu_b200 as sme
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    g = engine_graph(args)
    n, m, dmax = g.info()
    rp, cl = g.csr()
    digest = csr_digest(rp, cl)
    g.to_device(local)
    steps = make_steps(rp, args, args.warmup + args.steps)
    tune = {"warp_granularity": args.granularity, "list_only": int(args.list_only)}

    # L2 (126 MB) is flushed before every step by writing a 256 MiB buffer, so
    # no step starts with the previous step's lists in cache
    flush_buf = None if args.no_l2_flush else torch.empty(64 << 20, dtype=torch.int32, device=f"cuda:{local}")

    def flush_l2():
        if flush_buf is not None:
            flush_buf.fill_(1)
        torch.cuda.synchronize()

    def step(i, gr=g):
        q, roots = steps[i]
        flush_l2()
        c = gr.count(q, args.algo, roots=roots, device=local, **tune)
        return c, sme.last_stats()

    # the sampler runs from the warm-up on; the timed window's own samples are
    # reported when there are enough of them (the timed steps take tens of ms)
    clocks = ClockSampler(local)
    clocks.start()
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark_start()
    total_inst, dev_ms, kern_ms, alg_bytes, hot, launches = 0, 0.0, 0.0, 0, 0, 0
    per_q, counts = {}, {}
    for i in range(args.warmup, args.warmup + args.steps):
        c, s = step(i)
        counts[i] = c
        total_inst += c
        dev_ms += s.device_ms
        kern_ms += s.kernel_ms
        alg_bytes += s.algorithmic_bytes
        hot += s.hot_launches
        launches += s.kernel_launches
        e = per_q.setdefault(steps[i][0], [0, 0.0, 0])
        e[0] += c
        e[1] += s.device_ms / 1e3
        e[2] += 1
    torch.cuda.synchronize()
    clocks.mark_end()
    clk = clocks.stop()
    dev_ms_max, inst_all = reduce_over_ranks(dev_ms, total_inst, dist, "cuda")
    value = inst_all / (dev_ms_max / 1e3)

    # every timed step recounted by a second plan, outside the timed region
    check = {"plan": f"algo {args.check_algo}", "steps": 0, "equal": True}
    for i in counts:
        q, roots = steps[i]
        c2 = g.count(q, args.check_algo, roots=roots, device=local)
        check["steps"] += 1
        check["equal"] = check["equal"] and c2 == counts[i]

    # end to end through the C-ABI: the graph in host memory, copied to the
    # device every step (packed lists by default, the uint32 CSR beside it)
    e2e = None
    if not args.no_e2e:
        prp = torch.from_numpy(rp).pin_memory()
        pcl = torch.from_numpy(cl).pin_memory()
        gh = sme.Graph.from_csr(prp.numpy(), pcl.numpy(), copy=False)

        def e2e_run():
            e_inst, e_t, h2d, d2h = 0, 0.0, 0, 0
            q, roots = steps[0]
            gh.count(q, args.algo, roots=roots, device=local, **tune)
            for i in range(args.warmup, args.warmup + args.steps):
                q, roots = steps[i]
                flush_l2()
                t0 = time.perf_counter()
                c = gh.count(q, args.algo, roots=roots, device=local, **tune)
                e_t += time.perf_counter() - t0
                if c != counts[i]:
                    raise RuntimeError(f"end-to-end count {c} != device-resident count {counts[i]} at step {i}")
                e_inst += c
                s = sme.last_stats()
                h2d += s.h2d_bytes
                d2h += s.d2h_bytes
            return e_inst * world / e_t, h2d // args.steps, d2h // args.steps

        plain_value, plain_h2d, _ = e2e_run()
        pack_t0 = time.perf_counter()
        packed_bytes = gh.pack() if not args.no_pack else 0
        pack_s = time.perf_counter() - pack_t0
        value_e, h2d_e, d2h_e = e2e_run() if packed_bytes else (plain_value, plain_h2d, 8)
        e2e = {"value": value_e, "unit": UNIT, "h2d_bytes_per_step": h2d_e, "d2h_bytes_per_step": d2h_e,
               "packed": bool(packed_bytes),
               "plain_csr": {"value": plain_value, "h2d_bytes_per_step": plain_h2d},
               "pack_once_s": round(pack_s, 3) if packed_bytes else None,
               "counts_equal_resident": True,
               "note": "wall clock around each sme_count on a graph that is not resident: every step uploads "
                       "the graph from pinned host memory into the call's arena (the packed lists of "
                       "sme_graph_pack, expanded on the device, or the plain uint32 CSR in plain_csr), builds "
                       "the hub bitmaps, copies the step's root list and reads the count back"}
        del gh

    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else 0.0
    tr = load_traffic()
    alg_per_launch = alg_bytes // max(hot, 1)
    traffic = None
    if tr and "dram_per_algorithmic_byte" in tr:
        traffic = int(alg_per_launch * tr["dram_per_algorithmic_byte"])
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "intersection kernels (COMPUTE / COMPUTE_COUNT / COMPUTE_PATH_COUNT)",
                "algorithmic_bytes_per_launch": alg_per_launch, "avg_launch_ms": kern_ms / max(hot, 1),
                "launches": hot,
                "bytes_definition": "per path: 12 per backward list (row pointers + gathered vertex) + 4 x clipped "
                                    "pivot length x lists intersected + 4 per candidate written",
                "traffic": traffic,
                "dram_achieved_gbs": (round(traffic / (kern_ms / max(hot, 1) / 1e3) / 1e9, 1)
                                      if traffic and kern_ms > 0 else None),
                "dram_frac": (round(traffic / (kern_ms / max(hot, 1) / 1e3) / 1e9 / peak, 4)
                              if traffic and kern_ms > 0 else None),
                "traffic_source": tr.get("source") if tr else None,
                "note": "achieved/frac count the bytes the probe-based intersection must touch (4 per probed "
                        "word); DRAM moves 32-byte sectors, so physical traffic (traffic, dram_achieved_gbs, "
                        "dram_frac) is the ncu-measured multiple of them"}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        timed_steps = [steps[i] for i in range(args.warmup, args.warmup + args.steps)]
        try:
            cb = cpu_baseline(args, g, timed_steps, [counts[i] for i in range(args.warmup, args.warmup + args.steps)])
            cb["per_query_ratio"] = {q: (per_query_summary(per_q)[q]["value"] / v["value"] if v["value"] else None)
                                     for q, v in cb["per_query"].items()}
        except Exception as ex:  # reported in the line, never dropped silently
            cb = {"error": f"{type(ex).__name__}: {ex}"}
    legs = {}
    if rank == 0 and world == 1:
        if not args.no_whole:
            legs["whole_graph"] = bench_whole_graph(args, g, local, tune, peak)
        g.release_device()
        if not args.no_forms:
            for name, fn in (("batched", bench_batched), ("served", bench_served)):
                try:
                    legs[name] = fn(args, local)
                except Exception as ex:
                    legs[name] = {"error": f"{type(ex).__name__}: {ex}"}
            try:
                legs["noalloc"] = bench_noalloc(local)
            except Exception as ex:
                legs["noalloc"] = {"error": f"{type(ex).__name__}: {ex}"}
        if not args.no_s22:
            try:
                legs["s22"] = bench_s22(args, local, tune, peak)
            except Exception as ex:
                legs["s22"] = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        cfg = config_of(args, n, m, digest)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic", "config": cfg,
            "per_query": per_query_summary(per_q), "counts_checked": check,
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk, "gpu_launches": launches,
            "step_counts": [int(counts[i]) for i in sorted(counts)], "max_degree": dmax, **legs,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
