"""The graphs the reference's own build was run on (tests/golden/ref_counts.json).

Each graph comes from the engine's seeded host generators, then is put in the
canonical form the reference reads: both directions of every undirected edge,
no self-loops, no duplicates, sorted by (src, dst). The sha256 of that form is
stored beside the counts, so a generator change is caught before any count is
compared.

Sizes are kept inside the limits the reference's kernels were written for
(fixed shared-memory arrays): largest out-degree <= 300 under both
orientations, k <= 9 for binary encoding and k <= 7 for the list encoding
(kclique/kckernels_orientation.cuh:65-77, kclique/kckernels_pivoting.cuh:30).
"""
from __future__ import annotations

import hashlib

import numpy as np

# name -> (generator, arguments); planted cliques as (count, smin, smax, seed)
GRAPHS = {
    "er2000": ("er", (2000, 0.01, 1), None),            # the plain small configuration, seed 1
    "er300_planted24": ("er", (300, 0.08, 2), (1, 24, 24, 21)),
    "er400_dense": ("er", (400, 0.15, 7), None),
    "sbm600": ("sbm", (600, 4, 0.1, 0.005, 3), None),
    "rmat12": ("rmat", (12, 16.0, 0.57, 0.19, 0.19, 4), None),
    "chunglu20k": ("chunglu", (20000, 2.1, 10.0, 300.0, 5), (5, 20, 30, 51)),
    "complete24": ("complete", (24,), None),
    "triangle": ("edges", ([0, 1, 0], [1, 2, 2], 3), None),
}


def canonical(src, dst):
    """Both directions, no loops, no duplicates, sorted by (src, dst)."""
    s = np.asarray(src, dtype=np.int64)
    d = np.asarray(dst, dtype=np.int64)
    keep = s != d
    s, d = s[keep], d[keep]
    a = np.concatenate([s, d])
    b = np.concatenate([d, s])
    key = np.unique((a << 32) | b)
    return (key >> 32).astype(np.uint32), (key & 0xFFFFFFFF).astype(np.uint32)


def make(name: str):
    """(src, dst, n_nodes) of graph `name` in canonical form."""
    import kcgpu_b200 as kc

    kind, args, plant = GRAPHS[name]
    if kind == "edges":
        s, d, n = np.asarray(args[0], np.uint32), np.asarray(args[1], np.uint32), args[2]
    elif kind == "complete":
        i, j = np.triu_indices(args[0], 1)
        s, d, n = i.astype(np.uint32), j.astype(np.uint32), args[0]
    else:
        gen = {"er": kc.gen_er, "sbm": kc.gen_sbm, "chunglu": kc.gen_chung_lu}
        if kind == "rmat":
            sc, ef, a, b, c, seed = args
            el = kc.gen_rmat(sc, ef, a, b, c, seed=seed)
        else:
            el = gen[kind](*args)
        if plant:
            el.plant_cliques(*plant)
        s, d, n = el.arrays()
    cs, cd = canonical(s, d)
    return cs, cd, int(n)


def sha(src, dst) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(src, np.uint32).tobytes())
    h.update(np.ascontiguousarray(dst, np.uint32).tobytes())
    return h.hexdigest()


def write_bel(path, src, dst) -> None:
    """The reference's binary edge list: 24-byte records {dst u64, src u64,
    weight u64} (include/FIleReader.cuh:84-90)."""
    rec = np.zeros((len(src), 3), np.uint64)
    rec[:, 0] = dst
    rec[:, 1] = src
    rec.tofile(path)
