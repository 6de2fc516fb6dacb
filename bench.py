#!/usr/bin/env python
"""Benchmark of the batched k-clique engine on B200.

Workload (the batched configuration): 10,000 independent seeded graphs,
n log-uniform in [50, 5000], families ER (p ~ U[0.005, 0.05]), 4-block SBM
(p_in 0.1, p_out 0.005) and ER + one planted clique of size 20-40, k uniform
in [4, 12]; degree orientation; mode / unit / partition / encoding picked per
graph by the engine's autotuner. One step = counting every graph of the
batch exactly (CSR build, orientation and the captured counting launch).

  value   graphs/s with the edge lists already in HBM (device-input API);
  e2e     the same through the host API with page-locked host inputs,
          host->device copies and the read-back of the counts inside the step;
  plain   graphs/s of the one-graph-per-launch path on a sample of the batch;
  cpu_baseline  the CPU oracle (OpenMP, all host threads) on a bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
Under torchrun each rank counts its own batch (seed shifted by rank): weak
scaling, no collective on the data path; the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "graphs/s, batched exact k-clique counts (10,000 mixed small graphs, k 4-12)"
UNIT = "graphs/s"
# DRAM bytes (read + write) per input edge of one step's counting launches and
# of its build (CSR, orientation, queue) launches, from the ncu capture of the
# first 1,500 graphs of the batch (53,548,148 input edges) summarised in the
# file named below; a step's traffic is scaled from it by its input edges
# (both grow with the edges: the gather with the out-lists, the build with the
# pairs it reads and the CSR it writes).
DRAM_CAPTURE_EDGES = 53_548_148
COUNT_DRAM_BYTES_CAPTURED = 298.2e6 + 1.7e6
BUILD_DRAM_BYTES_CAPTURED = 6.21e9
DRAM_SOURCE = ("profiles/build_kernels_batched1500_dram.md (ncu dram__bytes_read.sum + dram__bytes_write.sum, "
               "1,500-graph capture scaled by input edges)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--graphs", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--plain-sample", type=int, default=400)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="batched", choices=["batched", "serving", "rmat", "chunglu", "er"])
    ap.add_argument("--scale", type=int, default=20, help="rmat: log2 of the vertex count")
    ap.add_argument("--ks", default="", help="single-graph legs: comma-separated k values")
    ap.add_argument("--unit", default="", help="single-graph legs: node|edge (default: the config's)")
    ap.add_argument("--part", type=int, default=-1, help="single-graph legs: partition size (default: the config's)")
    ap.add_argument("--time-limit", type=float, default=900.0,
                    help="single-graph legs: device time limit of one count in seconds (the count then reports "
                         "a timeout instead of a number)")
    ap.add_argument("--requests", type=int, default=2048)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--serve-max-edges", type=float, default=1e5)
    ap.add_argument("--streams", type=int, default=2, help="serving: worker contexts / streams")
    ap.add_argument("--no-serving", action="store_true", help="batched workload: skip the serving leg")
    ap.add_argument("--tune-sample", type=int, default=1500, help="batched: graphs of the autotuner comparison")
    ap.add_argument("--batch-chunk-edges", type=int, default=0,
                    help="batched e2e: pipeline chunk size in edges (0 = the library default, -1 = one pass)")
    ap.add_argument("--tune-time-limit", type=float, default=5.0,
                    help="batched: device seconds per counting pass in the autotuner comparison")
    return ap.parse_args()


def serving_requests(kc, n_req: int, seed: int, max_edges: float = 1e5):
    """Seeded request stream: R-MAT graphs with edges log-uniform in
    [1e3, max_edges] (scale = ceil(log2(E/16)), edge factor E / 2^scale), k
    uniform in 3..15, 30% of the requests asking about one of 8
    device-resident graphs. Exact counts of 15-cliques in multi-million-edge
    R-MAT graphs take hours on any hardware, so the edge range is capped."""
    rng = np.random.default_rng(seed)
    resident = []
    for i in range(8):
        E = int(np.exp(rng.uniform(np.log(1e3), np.log(max_edges))))
        scale = max(1, int(np.ceil(np.log2(E / 16))))
        resident.append(kc.gen_rmat(scale, E / (1 << scale), seed=seed * 1000 + i).arrays())
    reqs = []
    for r in range(n_req):
        k = int(rng.integers(3, 16))
        if rng.random() < 0.3:
            reqs.append(("resident", int(rng.integers(len(resident))), k))
        else:
            E = int(np.exp(rng.uniform(np.log(1e3), np.log(max_edges))))
            scale = max(1, int(np.ceil(np.log2(E / 16))))
            reqs.append(("oneshot", kc.gen_rmat(scale, E / (1 << scale), seed=seed * 1000 + 100 + r).arrays(), k))
    return resident, reqs


def spec_label(c: dict) -> str:
    """The reference's -q spelling of a method plus the unit ("p8b-node");
    partition 0 (each size class sizes its own) prints as A."""
    return "%s%s%s-%s" % ("opa"[c["mode"]], c["part"] if c["part"] else "A", "bn"[c["encoding"]],
                          ("node", "edge")[c["unit"]])


def autotune_leg(kc, ctx, s, d, off, nn, kk, choice, args):
    """The autotuner's choices on the batch (histogram), and the counting stage
    of a bounded sample of the batch (its first graphs) under the autotuner and
    under fixed methods: the sweep's best fixed method and the reference's
    two partition-8 bitmap methods. Device ms of the counting stage from the
    batch statistics; a method past the device time limit reports null."""
    from collections import Counter

    hist = Counter(spec_label(c) for c in choice)
    P = min(len(nn), args.tune_sample)
    a, b = 0, int(off[P])
    ss, dd, oo = s[a:b], d[a:b], off[:P + 1]
    sweep = {}
    try:
        sweep = json.loads((ROOT / "kcgpu_b200" / "autotune_sweep.json").read_text())
    except (OSError, ValueError):
        pass
    fixed = {"o8b-node": {"mode": "orient", "unit": "node", "part": 8, "encoding": "bitmap"},
             "p8b-node": {"mode": "pivot", "unit": "node", "part": 8, "encoding": "bitmap"}}
    # and the fixed methods the sweep timed on its whole sample
    bf = sweep.get("best_fixed_method")
    for name in [bf] + [n for n in sweep.get("whole_sample_ms", {}) if n != "table"]:
        if not name or name in fixed:
            continue
        code, unit = name.split("-")
        fixed[name] = {"mode": {"o": "orient", "p": "pivot", "a": "auto"}[code[0]], "unit": unit,
                       "part": 0 if code[1:-1] == "A" else int(code[1:-1]),
                       "encoding": "bitmap" if code[-1] == "b" else "list"}
    runs = {}
    ctx.set_time_limit(int(args.tune_time_limit * 1e9))
    try:
        for name, fx in [("autotuned", None)] + list(fixed.items()):
            try:
                best = None
                for _ in range(2):
                    _, st = kc.batch_count(ctx, ss, dd, oo, nn[:P], kk[:P], orientation="degree",
                                           autotune=fx is None, fixed=fx, return_stats=True)
                    best = st["ms_count"] if best is None else min(best, st["ms_count"])
                runs[name] = {"ms_count": best, "graphs_per_s_count_stage": P / (best / 1e3)}
            except kc.KCError as e:
                if e.name != "KC_ERR_DEVICE_TIMEOUT":
                    raise
                runs[name] = {"ms_count": None, "timeout_s": args.tune_time_limit}
    finally:
        ctx.set_time_limit(0)
    done = [v["ms_count"] for k, v in runs.items() if k != "autotuned" and v["ms_count"] is not None]
    return {"choice_histogram": dict(hist.most_common()), "sample": f"first {P} graphs of the batch",
            "counting_stage": runs, "sweep_best_fixed": bf, "sweep_decision": sweep.get("decision"),
            "tuned_over_best_fixed": (min(done) / runs["autotuned"]["ms_count"]) if done else None}


def run_serving(args):
    """The serving configuration on its own (one JSON line)."""
    import torch

    import kcgpu_b200 as kc

    torch.cuda.set_device(0)
    ctx = kc.Context(0)
    line = serving_leg(kc, ctx, args)
    print(json.dumps(line), flush=True)
    ctx.close()


def serving_leg(kc, ctx, args):
    """Continuous batching: requests arrive by a Poisson process at args.rate
    per second and are submitted as they arrive; latency = done - submission
    (server clock). The same requests then run one per call on the plain path
    in arrival order; both sets of counts must agree exactly."""
    resident, reqs = serving_requests(kc, args.requests, args.seed, args.serve_max_edges)
    rng = np.random.default_rng(args.seed + 1)
    gaps = rng.exponential(1.0 / args.rate, size=len(reqs))
    clocks = Clocks(0)
    with kc.Server(ctx, streams=args.streams, orientation="degen") as srv:
        ids = [srv.put_graph(s, d, n) for s, d, n in resident]

        def submit(kind, g, k):
            return srv.submit(ids[g], k) if kind == "resident" else srv.submit_edges(g[0], g[1], g[2], k)

        # warm-up, untimed: the whole request set once, all at once (every
        # worker's kernels, streams and device memory in use before timing)
        for t in [submit(kind, g, k) for kind, g, k in reqs]:
            srv.wait(t)
        clocks.start()
        t0 = time.perf_counter()
        tickets, arrive = [], []
        t_next = t0
        for (kind, g, k), gap in zip(reqs, gaps):
            t_next += gap
            while time.perf_counter() < t_next:
                time.sleep(max(0.0, min(0.0005, t_next - time.perf_counter())))
            arrive.append(time.perf_counter())
            tickets.append(submit(kind, g, k))
        results = [srv.wait(t) for t in tickets]
        t_end = time.perf_counter()
        clk = clocks.stop()
        # capacity: the same requests submitted all at once (the Poisson run
        # cannot go faster than its arrivals)
        t2 = time.perf_counter()
        cap_counts = [srv.wait(t)["count"] for t in [submit(kind, g, k) for kind, g, k in reqs]]
        capacity = len(reqs) / (time.perf_counter() - t2)
    # server timestamps are ms since the server started; turn them into
    # latencies from each request's own submission
    lat = [r["done_ms"] - r["submit_ms"] for r in results]
    served = len(reqs) / (t_end - t0)
    # plain path: the same requests one per call, in arrival order
    t1 = time.perf_counter()
    plain_counts = []
    for kind, g, k in reqs:
        s, d, n = resident[g] if kind == "resident" else g
        with kc.Graph.from_edges(ctx, s, d, n) as gr:
            gr.orient("degen")
            plain_counts.append(gr.count(k, mode="pivot", unit="node", part=0))
    t_plain = time.perf_counter() - t1
    exact = [r["count"] for r in results] == plain_counts and cap_counts == plain_counts
    return {"metric": "served graphs/s (Poisson %.0f req/s, R-MAT 1e3-%.0e edges, k 3-15)" % (args.rate, args.serve_max_edges),
            "value": served, "unit": "graphs/s", "n_gpus": 1, "higher_is_better": True,
            "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
            "plain": {"value": len(reqs) / t_plain, "unit": "graphs/s", "sample": "same requests, one per call"},
            "served_over_plain": served / (len(reqs) / t_plain), "bitexact": exact,
            "capacity": {"value": capacity, "unit": "graphs/s", "over_plain": capacity / (len(reqs) / t_plain),
                         "sample": "the same requests submitted all at once"},
            "config": {"workload": "serving: %d requests, 30%% on 8 resident graphs, degeneracy orientation, "
                                   "autotuned, %d worker streams" % (len(reqs), args.streams)},
            "clocks": clk, "data": "synthetic (seeded generators)"}


def run_single(args):
    """One of the single-graph configurations, counted by the plain one-graph
    path: the graph is built and oriented once, one untimed k = 3 count warms
    the kernels up, then each k is counted once; device time from the count
    statistics.
      er      : G(2000, 0.01) seed 1, degree orientation, orientation mode,
                node units, partition 8, bitmap, k = 4
      rmat    : R-MAT scale S, edge factor 16, (0.57, 0.19, 0.19), degeneracy,
                pivoting, edge units, partition 8, bitmap, k = 5, 7
      chunglu : Chung-Lu n = 4M, exponent 2.1, mean degree 20, cap 50k, 200
                planted cliques of 30-60, degeneracy, pivoting, node units,
                k = 3, 6, 9, 12
    Under torchrun (N > 1) every rank builds the whole graph and counts one
    unit shard of it (kc_count_shard); the counts are summed exactly over the
    ranks and the device time is the max over ranks (strong scaling)."""
    import torch

    import kcgpu_b200 as kc
    from kcgpu_b200 import sharding

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    ctx = kc.Context(local)
    shard = (rank, world) if world > 1 else None
    if args.workload == "er":
        el = kc.gen_er(2000, 0.01, 1)
        orient, mode, unit, part, ks, enc = "degree", "orient", "node", 8, [4], "bitmap"
        name = "ER G(2000, 0.01) seed 1"
    elif args.workload == "rmat":
        el = kc.gen_rmat(args.scale, 16, 0.57, 0.19, 0.19, seed=1)
        orient, mode, unit, part, ks, enc = "degen", "pivot", "edge", 8, [5, 7], "bitmap"
        name = "R-MAT scale %d, edge factor 16, (0.57,0.19,0.19,0.05), seed 1" % args.scale
    else:
        el = kc.gen_chung_lu(4_000_000, 2.1, 20.0, 50_000.0, 3)
        el.plant_cliques(200, 30, 60, 11)
        orient, mode, unit, part, ks, enc = "degen", "pivot", "node", 0, [3, 6, 9, 12], "bitmap"
        name = "Chung-Lu n=4M, exponent 2.1, mean degree 20, cap 50k, 200 planted cliques of 30-60"
    if args.ks:
        ks = [int(x) for x in args.ks.split(",")]
    if args.unit:
        unit = args.unit
    if args.part >= 0:
        part = args.part
    s, d, n = el.arrays()
    # exact counts of the same graph from the CPU oracle, when the fixture
    # file holds them (matched by the sha256 of the generated arrays)
    want = {}
    try:
        import hashlib

        h = hashlib.sha256()
        h.update(np.ascontiguousarray(s).tobytes())
        h.update(np.ascontiguousarray(d).tobytes())
        fx = json.loads((ROOT / "tests" / "golden" / "configs.json").read_text())["configs"]
        for rec in fx.values():
            if rec.get("input_sha256") == h.hexdigest() and isinstance(rec.get("counts"), dict):
                want = {int(k): int(v) for k, v in rec["counts"].items()}
    except (OSError, ValueError, KeyError):
        pass
    clocks = Clocks(local)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient(orient)
        info = g.info()
        rows = []
        g.count(3, mode=mode, unit=unit, part=part, encoding=enc)  # warm-up: loads and sizes every kernel
        ctx.set_time_limit(int(args.time_limit * 1e9))
        for k in ks:
            barrier(pg, local)
            clocks.start()
            t0 = time.perf_counter()
            try:
                r = g.count(k, mode=mode, unit=unit, part=part, encoding=enc, stats=True, shard=shard)
                ok = 1.0
            except kc.KCError as e:
                if e.name != "KC_ERR_DEVICE_TIMEOUT":
                    raise
                r, ok = None, 0.0
            # every rank takes the same collective steps, timeout or not
            ok = -max_over_ranks(pg, -ok, local)
            if not ok:
                clk = clocks.stop()
                clocks = Clocks(local)
                rows.append({"k": k, "count": None, "timeout_s": args.time_limit,
                             "wall_ms": (time.perf_counter() - t0) * 1e3, "clocks": clk})
                continue
            wall = time.perf_counter() - t0
            clk = clocks.stop()
            clocks = Clocks(local)
            ms = max_over_ranks(pg, r.stats["ms_total"], local)
            count = sharding.sum_u128(r.count) if pg is not None else r.count
            tree = int(max_over_ranks(pg, float(r.stats["tree_nodes"]), local))
            rows.append({"k": k, "count": str(count), "ms": ms, "wall_ms": wall * 1e3,
                         "kcliques_per_s": count / (ms / 1e3) if ms > 0 else None,
                         "tree_nodes" if pg is None else "tree_nodes_max_rank": tree,
                         "ms_launch": r.stats["ms_launch"],
                         "oracle_fixture": (count == want[k]) if k in want else None, "clocks": clk})
    line = {"metric": "single-graph k-clique counts (device ms per count)", "workload": args.workload,
            "n_gpus": world, "scaling": "strong" if world > 1 else None,
            "config": {"workload": name, "n": info["n"], "m": info["m"], "max_out_degree": info["max_out_degree"],
                       "orientation": orient, "mode": mode, "unit": unit, "part": part, "encoding": enc,
                       "parallelism": "unit shards over %d GPUs" % world if world > 1 else "single GPU"},
            "results": rows, "data": "synthetic (seeded generators)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(gpus: int, backend: str = "nccl"):
    """One process per GPU (torchrun env vars); the process group is only
    used for barriers and the max-over-ranks of the step time."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg, device):
    """device None: a host-only group (gloo)."""
    if pg is not None:
        if device is None:
            pg.barrier()
            return
        import torch

        pg.barrier(device_ids=[device])
        torch.cuda.synchronize()


def max_over_ranks(pg, x: float, device) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cpu" if device is None else f"cuda:{device}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def make_batch(kc, n_graphs: int, seed: int, pinned: bool = True):
    """The seeded batch; pageable batches come from the generator-only library,
    so a process that only runs the CPU reference never loads the engine."""
    el = kc.gen_batch(n_graphs, seed, pinned=True) if pinned else kc.gen_batch_host(n_graphs, seed)
    s, d, _ = el.arrays(copy=False)  # views of the generator's (page-locked when pinned) arrays
    off, nn, kk, fam = el.batch_meta()
    return el, s, d, off, nn, kk, fam


def cpu_modes(kk, fam):
    """The CPU counter's algorithm per graph: the Pivoter for graphs that hold
    a planted clique or ask for k >= 9, orientation listing for the rest (the
    faster of the two on the CPU for each family)."""
    return [1 if (int(k) >= 9 or int(f) == 2) else 0 for k, f in zip(kk, fam)]


def cpu_oracle_sample(s, d, off, nn, kk, modes, budget_s: float):
    """The CPU oracle on graphs 0, 1, ... until budget_s elapses; returns
    (graphs done, seconds, counts)."""
    from oracle.oracle import OracleGraph

    counts = []
    t0 = time.perf_counter()
    g = 0
    while g < len(nn) and time.perf_counter() - t0 < budget_s:
        a, b = int(off[g]), int(off[g + 1])
        og = OracleGraph(s[a:b], d[a:b], int(nn[g]))
        og.orient("degree")
        counts.append(og.count(int(kk[g]), mode="pivot" if modes[g] == 1 else "orient"))
        g += 1
    return g, time.perf_counter() - t0, counts


def run_reference(args, world, rank, local, pg):
    """The reference arm: KCGPU has no CPU counting path, so its CPU arm is the
    oracle port (OpenMP, every host thread) on a bounded sample per step."""
    if rank != 0:
        return
    import kcgpu_b200 as kc

    from oracle.oracle import max_threads

    el, s, d, off, nn, kk, fam = make_batch(kc, args.graphs, args.seed, pinned=False)
    modes = cpu_modes(kk, fam)
    # size one step to ~12 s of CPU work on this host
    probe, t_probe, _ = cpu_oracle_sample(s, d, off, nn, kk, modes, 3.0)
    per_graph = t_probe / max(1, probe)
    sample = int(max(1, min(args.graphs, 12.0 / max(per_graph, 1e-6))))
    times = []
    total = args.warmup + args.steps
    for i in range(total):
        done, dt, _ = cpu_oracle_sample(s, d, off[: sample + 1], nn[:sample], kk[:sample], modes, 1e9)
        if i >= args.warmup:
            times.append(dt)
    mean = sum(times) / len(times)
    val = sample / mean
    line = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64/u128 integer", "data": "synthetic (seeded)",
            "config": {"workload": "batched: first %d of %d mixed graphs (ER / 4-block SBM / ER+planted clique), "
                                   "n 50-5000, k 4-12, degree orientation" % (sample, args.graphs)},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": max_threads(), "kind": "port",
                             "sample": f"first {sample} graphs of the batch per step"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "serving" and args.impl == "engine":
        run_serving(args)
        return
    if args.workload in ("rmat", "chunglu", "er") and args.impl == "engine":
        run_single(args)
        return
    world, rank, local, pg = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    import torch

    torch.cuda.set_device(local)
    import kcgpu_b200 as kc

    ctx = kc.Context(local)
    ctx.set_batch_chunk_edges(2**64 - 1 if args.batch_chunk_edges < 0 else args.batch_chunk_edges)
    L = kc.lib()
    el, s, d, off, nn, kk, fam = make_batch(kc, args.graphs, args.seed + rank * args.graphs)
    G = len(nn)
    E = int(off[-1])
    d_s = torch.from_numpy(s.view(np.int32)).to(f"cuda:{local}")
    d_d = torch.from_numpy(d.view(np.int32)).to(f"cuda:{local}")
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=f"cuda:{local}")

    def run_device(with_choice=False):
        # the per-graph choices (10,000 dicts) are read once, after the timed steps
        r = kc.batch_count(ctx, None, None, off, nn, kk, orientation="degree", autotune=True, use_graph=True,
                           return_choice=with_choice, return_stats=True,
                           device_ptrs=(d_s.data_ptr(), d_d.data_ptr()))
        return r if with_choice else (r[0], None, r[1])

    def run_host():
        return kc.batch_count(ctx, s, d, off, nn, kk, orientation="degree", autotune=True, use_graph=True,
                              return_stats=True)

    for _ in range(args.warmup):
        counts, choice, st = run_device()
    # timed region: inputs (3 GB of edges) are larger than the 126 MB L2
    barrier(pg, local)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = L.kc_kernel_launches()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage = {"ms_h2d": [], "ms_build": [], "ms_csr": [], "ms_orient": [], "ms_count": [], "ms_host_total": []}
    trav = {"tree_nodes": 0, "word_ops": 0, "gather_bytes": 0, "heavy_units": 0}
    cycles = [0, 0, 0]
    host_ms = [0.0] * 5
    sizes = {}
    for i in range(args.steps):
        evs[i][0].record(stream)
        counts, choice, st = run_device()
        evs[i][1].record(stream)
        for key in stage:
            stage[key].append(st["ms_total" if key == "ms_host_total" else key])
        for key in trav:
            trav[key] += st[key]
        cycles = [a + b for a, b in zip(cycles, st["cycles"])]
        host_ms = [a + b / args.steps for a, b in zip(host_ms, st["host_ms"])]
        sizes = {"vertices": st["n_vertices"], "edges_dedup": st["n_edges"]}
    torch.cuda.synchronize()
    launches = (L.kc_kernel_launches() - l0) // max(1, args.steps)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    t_step = max_over_ranks(pg, sum(step_ms) / len(step_ms), local)
    value = world * G / (t_step / 1e3)

    # end to end through the host API: page-locked inputs, copies inside the step
    e2e_val = None
    if not args.no_e2e:
        counts_h = None
        for _ in range(args.warmup):  # the host path's own buffers (staging, copy stream)
            run_host()
        barrier(pg, local)
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            ev2[i][0].record(stream)
            counts_h, _ = run_host()
            ev2[i][1].record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(pg, sum(a.elapsed_time(b) for a, b in ev2) / args.steps, local)
        e2e_val = world * G / (e2e_ms / 1e3)
        assert counts_h == counts, "host-input and device-input batches disagree"

    _, choice, _ = run_device(with_choice=True)  # the autotuner's choices, untimed
    total_cliques = sum(counts)
    out = None
    if rank == 0:
        modes = cpu_modes(kk, fam)
        # plain path: one graph per call on a sample of the same batch
        P = min(args.plain_sample, G)
        t0 = time.perf_counter()
        plain_counts = []
        for g in range(P):
            a, b = int(off[g]), int(off[g + 1])
            with kc.Graph.from_edges(ctx, s[a:b], d[a:b], int(nn[g])) as gr:
                gr.orient("degree")
                c = choice[g]
                plain_counts.append(gr.count(int(kk[g]), mode=c["mode"], unit=c["unit"], part=c["part"],
                                             encoding=c["encoding"]))
        t_plain = time.perf_counter() - t0
        plain_gps = P / t_plain
        bitexact_plain = plain_counts == counts[:P]
        cpu = None
        bitexact_cpu = None
        if world == 1:
            from oracle.oracle import max_threads

            done, dt, ccounts = cpu_oracle_sample(s, d, off, nn, kk, modes, args.cpu_seconds)
            bitexact_cpu = ccounts == counts[:done]
            cpu = {"value": done / dt, "unit": UNIT, "cores": max_threads(), "kind": "port",
                   "sample": f"first {done} graphs of the batch, {dt:.1f} s, CPU oracle (OpenMP)",
                   "bitexact": bitexact_cpu}
        # the serving configuration, bounded (a few seconds), on this GPU
        serving = None if (args.no_serving or world > 1) else serving_leg(kc, ctx, args)
        tuning = autotune_leg(kc, ctx, s, d, off, nn, kk, choice, args)
        h2d = 8 * E + 8 * (G + 1) + 8 * G
        ms_count = sum(stage["ms_count"]) / len(stage["ms_count"])
        ms_build = sum(stage["ms_build"]) / len(stage["ms_build"])
        peaks = {}
        try:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        except (OSError, ValueError):
            pass
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"
        steps = max(1, args.steps)
        # Counting launch (k_count_bitmap, every counting kernel of a step).
        # Its algorithmic HBM bytes are the out-lists gathered to build the
        # induced subgraphs, 4 (|S| + sum of |N+(v)| over v in S) per unit,
        # counted by the kernels; DRAM traffic per step comes from the ncu
        # capture summarised in profiles/ (most of the gather hits L2).
        gb_s = (trav["gather_bytes"] / steps) / (ms_count / 1e3) / 1e9
        sm_mhz = (clk.get("sm_mhz") or 1965.0)
        popc_peak = 16 * 148 * sm_mhz * 1e6
        wops = (trav["word_ops"] / steps) / (ms_count / 1e3)
        tot_cy = max(1.0, float(sum(cycles)))
        roofline = {"bound": "hbm", "kernel": "k_count_bitmap (all counting launches of a step)",
                    "achieved": gb_s, "peak": hbm_peak, "unit": "GB/s", "frac": gb_s / hbm_peak,
                    "peak_source": peak_src, "algorithmic_bytes_per_step": trav["gather_bytes"] / steps,
                    "traffic": COUNT_DRAM_BYTES_CAPTURED * E / DRAM_CAPTURE_EDGES,
                    "traffic_source": DRAM_SOURCE,
                    "limiter": "not HBM: latency and integer issue of the gather and traversal (roofline_issue)"}
        # The same launch against its real limiter: where its unit groups spend
        # their cycles, and its AND+POPC word-operation rate against the POPC
        # issue rate (16 per SM per clock at the sampled SM clock).
        roofline_issue = {"bound": "int-issue", "kernel": "k_count_bitmap", "achieved": wops, "peak": popc_peak,
                          "unit": "word-ops/s", "frac": wops / popc_peak,
                          "group_cycle_share": {"form_S": cycles[0] / tot_cy, "gather_subgraph": cycles[1] / tot_cy,
                                                "traverse": cycles[2] / tot_cy},
                          "tree_nodes_per_step": trav["tree_nodes"] / steps,
                          "heavy_units_per_step": trav["heavy_units"] / steps}
        # CSR build + orientation: algorithmic bytes = read the input pairs
        # (8 E), write the symmetric CSR (8 m + 4 (n + 1)), read it again for the
        # orientation (8 m + 4 (n + 1)) and write the DAG (4 m + 4 (n + 1)).
        nv, mm = sizes.get("vertices", 0), sizes.get("edges_dedup", 0)
        build_bytes = 8 * E + 20 * mm + 12 * (nv + 1)
        roofline_build = {"bound": "hbm", "kernel": "CSR build + degree orientation (csr.cu, prims.cu, orient.cu)",
                          "achieved": build_bytes / (ms_build / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                          "frac": build_bytes / (ms_build / 1e3) / 1e9 / hbm_peak, "peak_source": peak_src,
                          "algorithmic_bytes_per_step": build_bytes,
                          "traffic": BUILD_DRAM_BYTES_CAPTURED * E / DRAM_CAPTURE_EDGES, "traffic_source": DRAM_SOURCE,
                          "ms": {"csr": sum(stage["ms_csr"]) / steps, "orient": sum(stage["ms_orient"]) / steps}}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64/u128 integer", "data": "synthetic (seeded generators)",
            "config": {"workload": "batched: %d mixed graphs (ER p~U[.005,.05] / 4-block SBM 0.1,0.005 / ER+planted "
                                   "clique 20-40), n log-uniform 50-5000, k U{4..12}, degree orientation, autotuned, "
                                   "one captured counting launch" % G,
                       "graphs": G, "edges": E, "l2": "inputs (%.1f GB) larger than L2" % (8 * E / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "kcliques_per_s": world * total_cliques / (t_step / 1e3),
            "plain": {"value": plain_gps, "unit": UNIT, "sample": f"first {P} graphs, one graph per call",
                      "bitexact": bitexact_plain},
            "batched_over_plain": value / plain_gps,
            "stage_ms": {k: sum(v) / len(v) for k, v in stage.items()},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16 * G + 24 * G},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
            "roofline": roofline,
            "roofline_issue": roofline_issue,
            "roofline_build": roofline_build,
            "serving": serving,
            "autotune": tuning,
            "host_ms": {"checks_h2d": host_ms[0], "build": host_ms[1], "plan": host_ms[2], "count": host_ms[3],
                        "readback": host_ms[4]},
        }
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
