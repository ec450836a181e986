#!/usr/bin/env python3
"""Benchmark of the GPU subgraph-enumeration path (one JSON line on rank 0).

Workload (the plain GPU path of the 4-clique / 4-cycle / diamond
configuration): an undirected R-MAT graph, scale 20, edge factor 16,
a/b/c/d = .57/.19/.19/.05, seeded, self loops and parallel edges removed,
uint32 CSR; queries 4-clique (Q3), 4-cycle (Q1) and diamond (Q2) with the
reference's symmetry-breaking constraints, counted with uint64 results by the
LIGHT plan in IN_MEMORY_GPU mode (`patternmatchgpu -a 6 -m 1`).

A step is one pass of the hot path over one task: the count of one query
over one root-vertex range of the graph (an IntraPartScheduler task).  The
steps cycle through (query, task) pairs; the sum over a full cycle is the
complete count of every query.  `value` is instances/s with the graph
resident in HBM, timed with CUDA events on the library's stream; `e2e` is the
same metric through sme_count with the CSR in pinned host memory copied to the
device in every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sme|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "instances/sec (4-clique, 4-cycle, diamond; R-MAT s20 ef16)"
UNIT = "instances/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=9)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sme", choices=["sme", "reference"])
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=20)
    ap.add_argument("--queries", default="3,1,2")
    ap.add_argument("--algo", type=int, default=6)
    ap.add_argument("--tasks", type=int, default=2, help="root-range tasks per query")
    ap.add_argument("--q1-stride", type=int, default=1024, help="4-cycle: roots per strided task = n/stride")
    ap.add_argument("--q1-tasks", type=int, default=3, help="4-cycle: strided tasks in the step cycle")
    ap.add_argument("--root-end", type=int, default=0, help="restrict roots to [0, root_end) (profiling)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--granularity", type=int, default=0, help="0 auto, 1 warp per path, 2 flattened")
    ap.add_argument("--list-only", action="store_true", help="no hub bitmaps (comparison)")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
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
                "reasons": sorted(reasons), "samples": len(sm)}


def make_graph(args):
    import subgraphmatchgpu_b200 as sme
    return sme.Graph.rmat(args.scale, args.edge_factor, 0.57, 0.19, 0.19, seed=args.seed)


def work_items(args, n):
    """(query, root_begin, root_end, root_stride) tasks.  Queries whose full
    count fits a few seconds (4-clique, diamond) use `tasks` contiguous root
    ranges; the 4-cycle, whose full count at this scale takes minutes, uses
    strided tasks (every `q1_stride`-th root from offset k), each an unbiased
    1/q1_stride slice of the roots."""
    qs = [int(q) for q in args.queries.split(",")]
    end = args.root_end or n
    items = []
    for q in qs:
        if q == 1 and not args.root_end:
            items += [(q, k, end, args.q1_stride) for k in range(args.q1_tasks)]
        else:
            cuts = [end * i // args.tasks for i in range(args.tasks + 1)]
            items += [(q, a, b, 1) for a, b in zip(cuts, cuts[1:])]
    return items


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(g, items, budget_s):
    """The oracle port (C restatement of CPU_WCOJ, OpenMP, all host threads)
    on a strided root sample of the same graph and query mix."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as O
    rp, cl = g.csr()
    n = len(rp) - 1
    threads = os.cpu_count() or 1
    import numpy as np
    qs = sorted({it[0] for it in items})
    # roots in a seeded random order (hubs and tail alike), processed until the
    # per-query share of the budget runs out; roots cut short are discarded
    roots = np.random.default_rng(12345).permutation(n).astype(np.uint32)
    total_inst, total_t, done = 0, 0.0, {}
    for q in qs:
        inst, d, t = O.count_sample(rp, cl, q, roots, budget_s / len(qs), threads)
        total_inst += inst
        total_t += t
        done[q] = d
    return {"value": total_inst / total_t if total_t > 0 else 0.0, "unit": UNIT, "cores": threads,
            "kind": "port",
            "sample": f"CPU_WCOJ port, {threads} threads, roots of the same R-MAT graph in a seeded random order "
                      f"until {budget_s / len(qs):.1f}s per query; completed roots per query {done}; "
                      f"{total_inst} instances in {total_t:.2f}s"}, total_inst, total_t


def run_reference(args, rank, world):
    """CPU reference arm: the oracle port of CPU_WCOJ on the host cores."""
    if rank != 0:
        return
    g = make_graph(args)
    items = work_items(args, g.n)
    # one calibrated sample per step; warm-up steps run the same sample
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(g, items, per_step)
    inst, t = 0, 0.0
    for _ in range(args.steps):
        cb, i, dt = cpu_baseline(g, items, per_step)
        inst += i
        t += dt
    cb["value"] = inst / t if t > 0 else 0.0
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": f"R-MAT s{args.scale} ef{args.edge_factor} seed {args.seed}, queries "
                                   f"{args.queries}, CPU_WCOJ on host cores (bounded sample)"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import subgraphmatchgpu_b200 as sme
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    g = make_graph(args)
    n, m, dmax = g.info()
    g.to_device(local)
    items = work_items(args, n)
    tune = {"warp_granularity": args.granularity, "list_only": int(args.list_only)}

    def step(i):
        q, a, b, st = items[i % len(items)]
        c = g.count(q, args.algo, root_begin=a, root_end=b, root_stride=st, device=local, **tune)
        return c, sme.last_stats()

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    total_inst, dev_ms, kern_ms, alg_bytes, hot, launches = 0, 0.0, 0.0, 0, 0, 0
    per_query = {}
    for i in range(args.steps):
        c, s = step(args.warmup + i)
        total_inst += c
        dev_ms += s.device_ms
        kern_ms += s.kernel_ms
        alg_bytes += s.algorithmic_bytes
        hot += s.hot_launches
        launches += s.kernel_launches
        q = items[(args.warmup + i) % len(items)][0]
        per_query.setdefault(q, [0, 0.0])
        per_query[q][0] += c
        per_query[q][1] += s.device_ms
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        t = torch.tensor([dev_ms, total_inst], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        dev_ms_max, inst_all = float(tmax[0]), float(t[1])
    else:
        dev_ms_max, inst_all = dev_ms, float(total_inst)
    value = inst_all / (dev_ms_max / 1e3)

    # end to end through the C-ABI: CSR in pinned host memory, copied every step
    e2e = None
    if not args.no_e2e:
        rp, cl = g.csr()
        prp = torch.from_numpy(rp).pin_memory()
        pcl = torch.from_numpy(cl).pin_memory()
        gh = sme.Graph.from_csr(prp.numpy(), pcl.numpy(), copy=False)
        e_inst, e_t, h2d, d2h = 0, 0.0, 0, 0
        q, a, b, st = items[-1]
        gh.count(q, args.algo, root_begin=a, root_end=b, root_stride=st, device=local, **tune)
        for i in range(args.steps):
            q, a, b, st = items[(args.warmup + i) % len(items)]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e_inst += gh.count(q, args.algo, root_begin=a, root_end=b, root_stride=st, device=local, **tune)
            e_t += time.perf_counter() - t0
            s = sme.last_stats()
            h2d += s.h2d_bytes
            d2h += s.d2h_bytes
        e2e = {"value": e_inst * world / e_t, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
               "d2h_bytes_per_step": d2h // args.steps}
        del gh

    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else 0.0
    tr = load_traffic()
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "k_compute (intersection: COMPUTE / COMPUTE_COUNT)",
                "algorithmic_bytes_per_launch": alg_bytes // max(hot, 1),
                "avg_launch_ms": kern_ms / max(hot, 1),
                "traffic": tr.get("traffic_bytes_per_launch") if tr else None,
                "traffic_source": tr.get("source") if tr else None}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, _, _ = cpu_baseline(g, items, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": f"R-MAT s{args.scale} ef{args.edge_factor} (a,b,c)=(.57,.19,.19) seed "
                                   f"{args.seed}: n={n} m={m} max_degree={dmax}; queries {args.queries} "
                                   f"(Q3 4-clique, Q1 4-cycle, Q2 diamond), plan algo {args.algo} "
                                   f"(6=LIGHT), IN_MEMORY_GPU, {args.tasks} root tasks per query",
                       "l2": "inputs larger than L2 (CSR bytes %d)" % (8 * (n + 1) + 4 * m),
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "per_query": {str(q): {"instances": v[0], "device_ms": v[1]} for q, v in per_query.items()}},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
