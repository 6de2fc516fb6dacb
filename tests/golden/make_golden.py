"""Writes tests/golden/closed_form.json: k-clique counts known in closed form.

K_n has C(n, k) k-cliques; a complete multipartite graph with part sizes
(n_1, ..., n_r) has e_k(n_1, ..., n_r) (elementary symmetric polynomial).
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
    cases.append({"graph": {"kind": "multipartite", "sizes": sizes}, "orientation": "degree",
                  "counts": {str(k): str(e_k(sizes, k)) for k in range(3, len(sizes) + 2)}})
out = Path(__file__).resolve().parent / "closed_form.json"
out.write_text(json.dumps({"source": "closed form (math.comb, elementary symmetric polynomials)",
                           "cases": cases}, indent=1))
print(out)
