"""The CPU oracle against brute force, closed forms and the golden fixtures.

The reference ships no tests or fixtures; the known answers here are
closed-form (K_n, complete multipartite graphs, disjoint unions, edgeless
graphs) and brute-force enumeration of every small graph case.
"""
import itertools
import json
import math
import random
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import OracleGraph, binom
from tests import graphs as G

GOLDEN = Path(__file__).resolve().parent / "golden"
MODES = [(m, u) for m in ("orient", "pivot") for u in ("node", "edge")]


def test_complete_graphs_closed_form():
    for n in (1, 2, 3, 5, 9, 14):
        s, d = G.complete(n)
        g = OracleGraph(s, d, n)
        for o in ("degree", "degen"):
            g.orient(o)
            for k in range(1, n + 2):
                for m, u in MODES:
                    if u == "edge" and k == 1:
                        continue
                    assert g.count(k, m, u) == math.comb(n, k)


def test_every_small_graph_matches_brute_force():
    rng = random.Random(7)
    for trial in range(120):
        n = rng.randint(1, 8)
        p = rng.random()
        pairs = [(i, j) for i in range(n) for j in range(i + 1, n) if rng.random() < p]
        s = np.array([a for a, _ in pairs], np.uint32)
        d = np.array([b for _, b in pairs], np.uint32)
        ms, md = G.messy(s, d, n, trial)
        g = OracleGraph(ms, md, n)
        for o in ("degree", "degen"):
            g.orient(o)
            for k in range(1, 7):
                want = G.brute_kcliques(n, s, d, k)
                for m, u in MODES:
                    if u == "edge" and k == 1:
                        continue
                    assert g.count(k, m, u) == want, (trial, o, k, m, u)


def test_multipartite_and_union():
    for sizes in ([3, 3, 3], [5, 1, 4, 2], [2] * 7):
        s, d, n = G.multipartite(sizes)
        g = OracleGraph(s, d, n)
        g.orient("degen")
        for k in range(2, len(sizes) + 2):
            assert g.count(k, "pivot") == G.multipartite_kcliques(sizes, k)
            assert g.count(k, "orient", "edge") == G.multipartite_kcliques(sizes, k)
    parts = [G.complete(6) + (6,), G.multipartite([3, 2, 2]), G.complete(9) + (9,)]
    s, d, n = G.disjoint_union(parts)
    g = OracleGraph(s, d, n)
    g.orient("degree")
    for k in (2, 3, 4, 5):
        total = 0
        for ps, pd, pn in parts:
            h = OracleGraph(ps, pd, pn)
            h.orient("degree")
            total += h.count(k)
        assert g.count(k, "pivot", "edge") == total


def test_csr_symmetrise_dedup_and_orientation_rules():
    s = np.array([0, 1, 1, 2, 2, 3, 0], np.uint32)
    d = np.array([1, 0, 2, 2, 3, 0, 1], np.uint32)
    g = OracleGraph(s, d, 5)
    rp, ci = g.csr()
    assert rp.tolist() == [0, 2, 4, 6, 8, 8]
    assert ci.tolist() == [1, 3, 0, 2, 1, 3, 0, 2]
    assert g.m == 4
    g.orient("degree")  # all degrees 2: ties broken by id, u -> v iff u < v
    rp, ci = g.dag()
    assert rp.tolist() == [0, 2, 3, 4, 4, 4] and ci.tolist() == [1, 3, 2, 3]


def python_peel(n, rp, col, m):
    """Straight restatement of SingleGPU_Kcore::findKcoreIncremental_async
    (kcore/kcore.cuh:442-584) as driven by src/main.cu:169, for small graphs."""
    deg = [int(rp[v + 1] - rp[v]) for v in range(n)]
    prio = [2 * m] * n
    level = [0] * n
    removed = [False] * n
    todo, pr, L = n, 0, 0
    while todo > 0:
        cur = [v for v in range(n) if not removed[v] and deg[v] == L]
        while cur:
            todo -= len(cur)
            for v in cur:
                level[v] = L
            if todo == 0:
                break
            mark = set(cur)
            for v in cur:
                prio[v] = pr
                removed[v] = True
            nxt = []
            for v in cur:
                for u in col[rp[v]:rp[v + 1]]:
                    if u in mark or removed[u]:
                        continue
                    old = deg[u]
                    deg[u] -= 1
                    if old == L + 1:
                        nxt.append(u)
            cur = nxt
            pr += 1
        L += 1
    return prio, level


def test_degeneracy_peel_matches_restatement():
    rng = np.random.default_rng(3)
    for trial in range(40):
        n = int(rng.integers(2, 60))
        p = float(rng.random() * 0.4)
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(iu.size) < p
        s, d = iu[keep].astype(np.uint32), ju[keep].astype(np.uint32)
        g = OracleGraph(s, d, n)
        g.orient("degen")
        prio, lev = g.peel()
        rp, ci = g.csr()
        wp, wl = python_peel(n, rp.tolist(), ci.tolist(), g.m)
        assert prio.tolist() == wp and lev.tolist() == wl, trial
        core, mx = g.kcore()
        assert mx == max(wl)


def test_truss_support_small():
    s, d = G.complete(5)
    g = OracleGraph(s, d, 5)
    assert g.truss_support().tolist() == [3] * 10
    s, d, n = G.multipartite([2, 2, 2])
    g = OracleGraph(s, d, n)
    assert set(g.truss_support().tolist()) == {2}


def test_binomials_exact():
    for n in range(0, 140, 3):
        for r in range(0, n + 1, 5):
            assert binom(n, r) == math.comb(n, r) % (1 << 128)


def test_golden_fixtures():
    """Closed-form counts pinned in tests/golden/closed_form.json hold for the oracle."""
    import kcgpu_b200 as kc

    for path in [GOLDEN / "closed_form.json"]:
        data = json.loads(path.read_text())
        for case in data["cases"]:
            s, d, n = build_case(kc, case["graph"])
            g = OracleGraph(s, d, n)
            g.orient(case.get("orientation", "degree"))
            for k, want in case["counts"].items():
                assert g.count(int(k), "pivot") == int(want), (path.name, case["graph"], k)
            for k, want in case.get("local", {}).items():
                assert g.count_local(int(k)) == [int(x) for x in want], (path.name, case["graph"], k)


def build_case(kc, spec):
    kind = spec["kind"]
    if kind == "complete":
        s, d = G.complete(spec["n"])
        return s, d, spec["n"]
    if kind == "multipartite":
        return G.multipartite(spec["sizes"])
    if kind == "er":
        el = kc.gen_er(spec["n"], spec["p"], spec["seed"])
    elif kind == "rmat":
        el = kc.gen_rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    elif kind == "sbm":
        el = kc.gen_sbm(spec["n"], spec["blocks"], spec["p_in"], spec["p_out"], spec["seed"])
    elif kind == "chung_lu":
        el = kc.gen_chung_lu(spec["n"], spec["exponent"], spec["mean"], spec["cap"], spec["seed"])
    else:
        raise ValueError(kind)
    if "plant" in spec:
        pc = spec["plant"]
        el.plant_cliques(pc["count"], pc["smin"], pc["smax"], pc["seed"])
    return el.arrays()


def test_pivoter_deep_trees_any_thread_count():
    # Planted cliques of 25-35 vertices give drop chains deeper than the
    # Pivoter's first scratch allocation, so its per-depth scratch grows (and
    # moves) in the middle of the recursion; the count must not depend on
    # that or on the thread count, and must equal the orientation listing.
    import kcgpu_b200 as kc

    el = kc.gen_chung_lu(20_000, 2.1, 12.0, 500.0, 9)
    el.plant_cliques(4, 25, 35, 3)
    s, d, n = el.arrays()
    og = OracleGraph(s, d, n)
    og.orient("degen")
    for k in (5, 8):
        want = og.count(k, "orient")
        assert want >= 4 * math.comb(25, k)
        assert og.count(k, "pivot", threads=1) == want
        assert og.count(k, "pivot") == want
        assert og.count(k, "pivot", "edge") == want


def test_local_counts_brute_force():
    # every k-clique credits each of its vertices: brute force on small graphs,
    # sums equal k times the global count, complete graphs in closed form
    rng = random.Random(5)
    for trial in range(12):
        n = rng.randint(1, 14)
        p = rng.choice([0.2, 0.5, 0.8])
        edges = [(i, j) for i in range(n) for j in range(i + 1, n) if rng.random() < p]
        s = np.array([e[0] for e in edges], np.uint32)
        d = np.array([e[1] for e in edges], np.uint32)
        og = OracleGraph(s, d, n)
        og.orient("degen" if trial % 2 else "degree")
        adj = {(min(a, b), max(a, b)) for a, b in edges}
        for k in (1, 2, 3, 4, 5):
            want = [0] * n
            for c in itertools.combinations(range(n), k):
                if all((a, b) in adj for a, b in itertools.combinations(c, 2)):
                    for v in c:
                        want[v] += 1
            got = og.count_local(k)
            assert got == want, (trial, k)
            assert sum(got) == k * og.count(k)
    s, d = G.complete(9)
    og = OracleGraph(s, d, 9)
    og.orient("degree")
    assert og.count_local(4) == [math.comb(8, 3)] * 9


def test_pivoter_closed_form_nodes_equal_plain_expansion():
    """The oracle's closed form for clique-tree nodes with k - held <= 2 (used
    to make the full-size fixtures) gives the plain expansion's count."""
    import kcgpu_b200 as kc

    for seed in range(30):
        rng = np.random.default_rng(seed)
        n = int(rng.integers(5, 120))
        p = float(rng.uniform(0.05, 0.6))
        s, d, nn = kc.gen_er(n, p, seed).arrays()
        g = OracleGraph(s, d, nn)
        g.orient("degen" if seed % 2 else "degree")
        for k in range(1, 9):
            for unit in ("node", "edge"):
                if unit == "edge" and k == 1:
                    continue
                assert g.count(k, "pivot", unit) == g.count(k, "pivot", unit, closed=True), (seed, k, unit)
