"""Seeded test graphs shared by the CPU and GPU tests (edge lists as numpy)."""
from __future__ import annotations

import itertools
import math

import numpy as np


def complete(n: int, offset: int = 0):
    if n < 2:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    i, j = np.triu_indices(n, 1)
    return (i + offset).astype(np.uint32), (j + offset).astype(np.uint32)


def multipartite(sizes):
    """Complete multipartite (Turán-type) graph with the given part sizes."""
    offs = np.cumsum([0] + list(sizes))
    s, d = [], []
    for a in range(len(sizes)):
        for b in range(a + 1, len(sizes)):
            x, y = np.meshgrid(np.arange(offs[a], offs[a + 1]), np.arange(offs[b], offs[b + 1]), indexing="ij")
            s.append(x.ravel())
            d.append(y.ravel())
    if not s:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32), int(offs[-1])
    return np.concatenate(s).astype(np.uint32), np.concatenate(d).astype(np.uint32), int(offs[-1])


def multipartite_kcliques(sizes, k: int) -> int:
    """e_k(sizes): a k-clique picks one vertex from each of k distinct parts."""
    e = [1] + [0] * k
    for s in sizes:
        for j in range(k, 0, -1):
            e[j] += e[j - 1] * s
    return e[k]


def disjoint_union(parts):
    """parts: list of (src, dst, n); returns the union with shifted ids."""
    s, d, off = [], [], 0
    for a, b, n in parts:
        s.append(np.asarray(a, np.uint64) + off)
        d.append(np.asarray(b, np.uint64) + off)
        off += n
    return np.concatenate(s).astype(np.uint32), np.concatenate(d).astype(np.uint32), off


def brute_kcliques(n: int, src, dst, k: int) -> int:
    adj = [set() for _ in range(n)]
    for u, v in zip(src.tolist(), dst.tolist()):
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    if k == 1:
        return n
    return sum(1 for c in itertools.combinations(range(n), k)
               if all(b in adj[a] for a, b in itertools.combinations(c, 2)))


def relabel(src, dst, n: int, seed: int):
    perm = np.random.default_rng(seed).permutation(n).astype(np.uint32)
    return perm[src], perm[dst]


def messy(src, dst, n: int, seed: int):
    """Adds reversed duplicates and self-loops and shuffles the order."""
    rng = np.random.default_rng(seed)
    m = src.size
    pick = rng.integers(0, max(1, m), size=max(1, m // 3)) if m else np.zeros(0, np.int64)
    loops = rng.integers(0, max(1, n), size=3).astype(np.uint32) if n else np.zeros(0, np.uint32)
    s = np.concatenate([src, dst[pick], loops, src[pick]]).astype(np.uint32)
    d = np.concatenate([dst, src[pick], loops, dst[pick]]).astype(np.uint32)
    order = rng.permutation(s.size)
    return s[order], d[order]


def comb(n, k):
    return math.comb(n, k)
