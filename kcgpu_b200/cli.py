"""Command line of the engine, with the reference's flag surface.

    python -m kcgpu_b200.cli -g GRAPH -m kc -o degree|degen -k K -p node|edge -q o8b [-d DEV]

mirrors ``main.cu.exe -g <file> -d <dev> -m kc -o ... -k K -p ... -q ...``
(src/main.cu:263-588, flags parsed in include/Config.h:291-363) and prints the
reference's ``Counter = N`` line, with the exact count instead of one that
wraps at 2^64. ``-m lkc`` prints the per-vertex counts of the first 50
vertices as the reference's SingleGPU_Kclique_Local::show does
(src/main.cu:590-760, binary encoding); ``-m kcore``
prints the maximum core (src/main.cu:248-261).
``-w``, ``-s`` and ``-a`` are accepted and ignored: the engine keeps no
windows, sorts and deduplicates any input itself, and always allocates on the
device.

GRAPH is a file or a seeded generator:
  *.tsv / *.txt / *.el   one edge per line ("src dst [weight]"), lines that
                         start with '#' or '%' skipped, ids as given
  *.mtx                  Matrix Market coordinate file (1-based ids)
  *.bel                  24-byte records {dst u64, src u64, weight u64}
                         (include/FIleReader.cuh:84-90)
  gen:er:N:P:SEED
  gen:rmat:SCALE:EDGE_FACTOR:SEED          (a, b, c) = (0.57, 0.19, 0.19)
  gen:chunglu:N:EXPONENT:MEAN:CAP:SEED[:CLIQUES:SMIN:SMAX:CSEED]
"""
from __future__ import annotations

import argparse
import sys
import time

import kcgpu_b200 as kc


def read_graph(spec: str):
    """Returns (src, dst, n_nodes) as uint32 arrays."""
    if spec.startswith("gen:"):
        f = spec.split(":")[1:]
        kind = f[0]
        if kind == "er":
            el = kc.gen_er(int(f[1]), float(f[2]), int(f[3]))
        elif kind == "rmat":
            el = kc.gen_rmat(int(f[1]), float(f[2]), 0.57, 0.19, 0.19, seed=int(f[3]))
        elif kind == "chunglu":
            el = kc.gen_chung_lu(int(f[1]), float(f[2]), float(f[3]), float(f[4]), int(f[5]))
            if len(f) > 6:
                el.plant_cliques(int(f[6]), int(f[7]), int(f[8]), int(f[9]))
        else:
            raise SystemExit(f"unknown generator {kind!r}")
        return el.arrays()
    return kc.read_edgelist(spec).arrays()  # by extension: .bel, .mtx, else a text edge list


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="k-clique counting on one GPU (reference-compatible flags)")
    ap.add_argument("-g", required=True, help="graph file or gen:... spec")
    ap.add_argument("-d", type=int, default=0, help="CUDA device")
    ap.add_argument("-m", default="kc", choices=["kc", "lkc", "kcore"])
    ap.add_argument("-o", default="degree", choices=["degree", "degen"])
    ap.add_argument("-k", type=int, default=4)
    ap.add_argument("-p", default="node", choices=["node", "edge"])
    ap.add_argument("-q", default="o8b", help="[o|p]<part>[b|n]: orientation or pivoting, partition size, "
                                              "binary or list encoding")
    ap.add_argument("-w", default="0")
    ap.add_argument("-s", default="0")
    ap.add_argument("-a", default="gpu")
    a = ap.parse_args(argv)

    t0 = time.perf_counter()
    src, dst, n = read_graph(a.g)
    ctx = kc.Context(a.d)
    g = kc.Graph.from_edges(ctx, src, dst, n)
    g.orient(a.o)
    t1 = time.perf_counter()
    info = g.info()
    print(f"Graph: n = {info['n']}, m = {info['m']}, max degree = {info['max_degree']}, "
          f"max out-degree = {info['max_out_degree']}")
    print(f"Preprocess time = {t1 - t0:.6f} s")
    if a.m == "kcore":
        _, mx = g.kcore()
        print(f"Max core = {mx}")
    elif a.m == "lkc":
        spec = kc.parse_spec(a.q)
        t2 = time.perf_counter()
        cpn = g.count_local(a.k, unit=a.p, part=spec["part"], mode="pivot" if spec["mode"] == 1 else "orient")
        t3 = time.perf_counter()
        print(f"count time = {t3 - t2:.6f} s")
        print(f"Local clique counter for the first {min(50, len(cpn))} Nodes:")
        for v in range(min(50, len(cpn))):
            print(f"{v}\t{cpn[v]}")
    else:
        spec = kc.parse_spec(a.q)
        mode = "pivot" if spec["mode"] == 1 else "orient"
        enc = "list" if spec["encoding"] == 1 else "bitmap"
        t2 = time.perf_counter()
        c = g.count(a.k, mode=mode, unit=a.p, part=spec["part"], encoding=enc)
        t3 = time.perf_counter()
        print(f"Counter = {c}")
        print(f"count time = {t3 - t2:.6f} s")
    g.close()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
