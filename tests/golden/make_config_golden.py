"""Exact counts of the full-size benchmark configurations: tests/golden/configs.json.

The CPU oracle (oracle/oracle.cpp, OpenMP, no GPU) counts each configuration
once; the GPU tests compare the engine's counts with these numbers. Pivoting
runs use the oracle's closed form for clique-tree nodes with k - held <= 2
(the same count as the plain expansion, checked against it in
tests/test_oracle.py), which makes the large configurations feasible on a
CPU.

  plain_small   ER G(2000, 0.01) seed 1, degree orientation, k = 3, 4
  rmat20        R-MAT scale 20, edge factor 16, (0.57, 0.19, 0.19, 0.05), seed 1,
                degeneracy orientation, k = 5, 7
  rmat18        the same generator at scale 18, k = 5, 7
  chunglu4m     Chung-Lu n = 4M, exponent 2.1, mean degree 20, cap 50k, seed 3,
                + 200 planted cliques of 30-60 (seed 11), degeneracy, k = 3..12
                as far as the time budget allows
  batch10k      the 10,000-graph batch of bench.py (seed 20261203): every
                graph's count, plus the sha256 of the generated arrays

Each graph records the sha256 of the generator's output, so a changed
generator fails loudly instead of comparing different graphs. The file is
rewritten after every count, so an interrupted run keeps what it finished.

    python tests/golden/make_config_golden.py [--only name,...] [--budget SECONDS]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

OUT = HERE / "configs.json"
BATCH_SEED = 20261203
BATCH_GRAPHS = 10_000


def sha_arrays(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def graph_spec(name: str):
    """(generator description, src, dst, n, orientation, ks, mode)."""
    import kcgpu_b200 as kc

    if name == "plain_small":
        s, d, n = kc.gen_er(2000, 0.01, 1).arrays()
        return "gen_er(2000, 0.01, seed=1)", s, d, n, "degree", [3, 4], "orient"
    if name in ("rmat20", "rmat18"):
        sc = 20 if name == "rmat20" else 18
        s, d, n = kc.gen_rmat(sc, 16, 0.57, 0.19, 0.19, seed=1).arrays()
        return f"gen_rmat({sc}, 16, 0.57, 0.19, 0.19, seed=1)", s, d, n, "degen", [5, 7], "pivot"
    if name == "chunglu4m":
        el = kc.gen_chung_lu(4_000_000, 2.1, 20.0, 50_000.0, 3)
        el.plant_cliques(200, 30, 60, 11)
        s, d, n = el.arrays()
        return ("gen_chung_lu(4000000, 2.1, 20.0, 50000.0, seed=3) + plant_cliques(200, 30, 60, seed=11)", s, d, n,
                "degen", list(range(3, 13)), "pivot")
    raise KeyError(name)


def load() -> dict:
    if OUT.exists():
        return json.loads(OUT.read_text())
    return {"what": "exact k-clique counts of the benchmark configurations from the CPU oracle",
            "made_by": "tests/golden/make_config_golden.py", "configs": {}}


def save(fx: dict) -> None:
    OUT.write_text(json.dumps(fx, indent=1) + "\n")


def run_graph(fx: dict, name: str, budget: float) -> None:
    from oracle.oracle import OracleGraph, max_threads

    desc, s, d, n, orient, ks, mode = graph_spec(name)
    rec = fx["configs"].setdefault(name, {})
    rec.update({"generator": desc, "input_sha256": sha_arrays(s, d), "n_nodes": int(n), "input_edges": int(len(s)),
                "orientation": orient, "oracle_mode": mode, "threads": max_threads()})
    rec.setdefault("counts", {})
    rec.setdefault("oracle_seconds", {})
    og = OracleGraph(s, d, n)
    rec["m"] = og.m
    rec["max_out_degree"] = og.orient(orient)
    spent = 0.0
    last, prev = 0.0, 0.0
    for k in ks:
        if str(k) in rec["counts"]:
            prev, last = last, float(rec["oracle_seconds"].get(str(k), 0.0))
            continue
        # the cost grows with k: predict the next count from the growth of the
        # last two and stop when it would not fit the budget
        growth = max(2.0, last / prev) if prev > 0 else 4.0
        if last and spent + growth * last > budget:
            rec.setdefault("not_counted", []).append(k)
            continue
        t0 = time.perf_counter()
        c = og.count(k, mode, "node", closed=(mode == "pivot"))
        prev, last = last, time.perf_counter() - t0
        spent += last
        rec["counts"][str(k)] = str(c)
        rec["oracle_seconds"][str(k)] = round(last, 2)
        save(fx)
        print(f"{name} k={k}: {c} ({last:.1f} s)", flush=True)


def run_batch(fx: dict) -> None:
    import kcgpu_b200 as kc
    from oracle.oracle import OracleGraph, max_threads

    el = kc.gen_batch(BATCH_GRAPHS, BATCH_SEED)
    s, d, _ = el.arrays(copy=False)
    off, nn, kk, fam = el.batch_meta()
    rec = {"generator": f"gen_batch({BATCH_GRAPHS}, seed={BATCH_SEED})",
           "input_sha256": sha_arrays(s, d, off, nn, kk, fam), "orientation": "degree", "threads": max_threads()}
    counts = []
    t0 = time.perf_counter()
    for g in range(len(nn)):
        a, b = int(off[g]), int(off[g + 1])
        og = OracleGraph(s[a:b], d[a:b], int(nn[g]))
        og.orient("degree")
        piv = int(kk[g]) >= 9 or int(fam[g]) == 2  # planted clique or large k: the Pivoter
        counts.append(str(og.count(int(kk[g]), "pivot" if piv else "orient", closed=piv)))
        if g % 1000 == 999:
            print(f"batch: {g + 1} graphs, {time.perf_counter() - t0:.0f} s", flush=True)
    rec["counts"] = counts
    rec["oracle_seconds"] = round(time.perf_counter() - t0, 1)
    fx["configs"]["batch10k"] = rec
    save(fx)


def main():
    global OUT
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="plain_small,rmat18,rmat20,batch10k,chunglu4m")
    ap.add_argument("--budget", type=float, default=3600.0, help="oracle seconds per single-graph config")
    ap.add_argument("--out", default=str(OUT), help="fixture file (several runs can write separate files and "
                                                     "be merged with --merge)")
    ap.add_argument("--merge", default="", help="comma-separated fixture files whose configs are merged into --out")
    args = ap.parse_args()
    OUT = Path(args.out)
    fx = load()
    if args.merge:
        for f in args.merge.split(","):
            fx["configs"].update(json.loads(Path(f).read_text())["configs"])
        save(fx)
        return
    for name in args.only.split(","):
        if name == "batch10k":
            run_batch(fx)
        else:
            run_graph(fx, name, args.budget)
    save(fx)


if __name__ == "__main__":
    main()
