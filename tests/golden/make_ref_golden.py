"""Records the reference's own counts: tests/golden/ref_counts.json.

Runs the reference's k-clique program (KCGPU src/main.cu, built for sm_100a
by oracle/build_ref.sh into oracle/_ref/kcgpu_ref) on the graphs of
ref_graphs.py, under every method of its `-m kc` path: node and edge units
(-p), orientation and pivoting (-q o/p), binary and list encoding (-q b/n),
partition sizes (-q 1..32), degree and degeneracy orientation (-o), several
k. The count of a run is the last "Counter = N" line it prints
(kclique/kclique.cuh:1671-1672); a run that prints none had no unit with
enough out-degree and counted 0. Needs a GPU; run once, on a B200:

    python tests/golden/make_ref_golden.py --out gpurun_out/ref_counts.json

The graphs, the exact binomial table the pivot methods read (written in the
reference's format, 1001 x 401 comma-separated values, C(r, c) and 0 for
c > r) and the runs' logs stay in a temporary directory. The fixture keeps,
per graph, its generator arguments and the sha256 of its canonical edge list,
and per run the command-line method, k, the count and the reference's own
timings ("count time", "Preprocess time").
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import ref_graphs as rg  # noqa: E402

BIN = ROOT / "oracle" / "_ref" / "kcgpu_ref"
K_BINARY = (3, 4, 5, 6, 7, 9)   # node/orientation/binary counts to k <= 9 (six stack levels)
K_LIST = (3, 4, 5, 6, 7)        # list encoding keeps per-level flags in a char
PART_SWEEP_GRAPHS = ("er300_planted24", "rmat12")


def write_ncr(path: Path) -> None:
    with open(path, "w") as f:
        for r in range(1001):
            row = []
            for c in range(401):
                row.append(repr(float(math.comb(r, c))) if c <= r else "0")
            f.write(",".join(row) + ",\n")


def run_one(bel: Path, orient: str, unit: str, spec: str, k: int, env: dict, timeout: float) -> dict:
    cmd = [str(BIN), "-g", str(bel), "-d", "0", "-m", "kc", "-o", orient, "-k", str(k), "-p", unit, "-q", spec,
           "-w", "0"]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    wall = time.perf_counter() - t0
    out = r.stdout + r.stderr
    counters = re.findall(r"Counter = (\d+)", out)
    ct = re.findall(r"count time ([0-9.eE+-]+) s", out)
    pt = re.findall(r"Preprocess time: ([0-9.eE+-]+) s", out)
    rec = {"orient": orient, "unit": unit, "spec": spec, "k": k, "rc": r.returncode, "wall_s": round(wall, 3),
           "count": counters[-1] if counters else ("0" if r.returncode == 0 else None),
           "counter_lines": len(counters),
           "count_time_s": float(ct[-1]) if ct else None, "preprocess_s": float(pt[-1]) if pt else None}
    if r.returncode != 0 or "error" in out.lower() and not counters:
        rec["tail"] = out[-600:]
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "ref_counts.json"))
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--timeout", type=float, default=120.0)
    ap.add_argument("--graphs", default="", help="comma-separated subset of ref_graphs.GRAPHS")
    args = ap.parse_args()
    if not BIN.exists():
        sys.exit(f"{BIN} is missing: run bash oracle/build_ref.sh where the reference sources are")
    names = [g for g in (args.graphs.split(",") if args.graphs else rg.GRAPHS)]
    tmp = Path(tempfile.mkdtemp(prefix="kcref_"))
    ncr = tmp / "nCr.txt"
    write_ncr(ncr)
    env = dict(os.environ, LC_ALL="C", LANG="C", KC_REF_NCR=str(ncr))
    graphs, jobs = {}, []
    for name in names:
        s, d, n = rg.make(name)
        bel = tmp / f"{name}.bel"
        rg.write_bel(bel, s, d)
        graphs[name] = {"generator": list(map(str, rg.GRAPHS[name][:2])), "planted": rg.GRAPHS[name][2],
                        "n": n, "directed_entries": int(len(s)), "sha256": rg.sha(s, d)}
        specs = [("o8b", K_BINARY), ("p8b", K_BINARY), ("o8n", K_LIST), ("p8n", K_LIST)]
        for orient in ("degree", "degen"):
            for unit in ("node", "edge"):
                for spec, ks in specs:
                    for k in ks:
                        jobs.append((name, bel, orient, unit, spec, k))
        if name in PART_SWEEP_GRAPHS:
            for algo in "op":
                for part in (1, 2, 4, 16, 32):
                    for enc in "bn":
                        for unit in ("node", "edge"):
                            jobs.append((name, bel, "degree", unit, f"{algo}{part}{enc}", 5))
    runs = []
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=args.workers) as ex:
        futs = {ex.submit(run_one, j[1], j[2], j[3], j[4], j[5], env, args.timeout): j for j in jobs}
        for f in cf.as_completed(futs):
            j = futs[f]
            try:
                rec = f.result()
            except subprocess.TimeoutExpired:
                rec = {"orient": j[2], "unit": j[3], "spec": j[4], "k": j[5], "rc": None, "count": None,
                       "tail": "timed out"}
            rec["graph"] = j[0]
            runs.append(rec)
    runs.sort(key=lambda r: (r["graph"], r["orient"], r["unit"], r["spec"], r["k"]))
    fixture = {
        "what": "counts printed by the reference's own -m kc program (KCGPU src/main.cu) rebuilt for sm_100a",
        "binary": "oracle/_ref/kcgpu_ref (oracle/build_ref.sh)",
        "made_by": "tests/golden/make_ref_golden.py",
        "seconds": round(time.perf_counter() - t0, 1),
        "graphs": graphs,
        "runs": runs,
    }
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    Path(args.out).write_text(json.dumps(fixture, indent=0) + "\n")
    bad = [r for r in runs if r.get("rc") != 0]
    print(f"{len(runs)} runs, {len(bad)} failed, {fixture['seconds']} s -> {args.out}")


if __name__ == "__main__":
    main()
