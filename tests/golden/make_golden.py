"""Writes tests/golden/closed_form.json: k-clique counts known in closed form.

K_n has C(n, k) k-cliques; a complete multipartite graph with part sizes
(n_1, ..., n_r) has e_k(n_1, ..., n_r) (elementary symmetric polynomial).
Local (per-vertex) counts: a vertex of K_n is in C(n-1, k-1) of them, a vertex
of part i in e_{k-1} of the other parts' sizes.
Values come from Python integers, independent of the oracle and the engine.
Run: python tests/golden/make_golden.py
"""
import json
import math
from pathlib import Path


def e_k(sizes, k):
    e = [1] + [0] * k
    for s in sizes:
        for j in range(k, 0, -1):
            e[j] += e[j - 1] * s
    return e[k]


cases = []
for n in (4, 10, 33, 64, 100):
    cases.append({"graph": {"kind": "complete", "n": n}, "orientation": "degen",
                  "counts": {str(k): str(math.comb(n, k)) for k in (3, 4, 5, 7, n // 2, n)}})
for sizes in ([3, 3, 3], [5, 1, 4, 2], [10] * 6, [2] * 16):
    # local counts: a vertex of part i is in e_{k-1}(sizes without part i) k-cliques
    # (kept to k with at most 1e6 cliques: the oracle lists them one by one)
    local = {}
    for k in range(3, len(sizes) + 2):
        if e_k(sizes, k) > 10**6:
            continue
        per_part = [str(e_k(sizes[:i] + sizes[i + 1:], k - 1)) for i in range(len(sizes))]
        local[str(k)] = [per_part[i] for i, sz in enumerate(sizes) for _ in range(sz)]
    cases.append({"graph": {"kind": "multipartite", "sizes": sizes}, "orientation": "degree",
                  "counts": {str(k): str(e_k(sizes, k)) for k in range(3, len(sizes) + 2)},
                  "local": local})
for n in (4, 10, 33):
    cases[[c["graph"] for c in cases].index({"kind": "complete", "n": n})]["local"] = {
        str(k): [str(math.comb(n - 1, k - 1))] * n for k in (3, 4, 5, 7, n // 2, n) if math.comb(n, k) <= 10**6}
out = Path(__file__).resolve().parent / "closed_form.json"
out.write_text(json.dumps({"source": "closed form (math.comb, elementary symmetric polynomials)",
                           "cases": cases}, indent=1))
print(out)
