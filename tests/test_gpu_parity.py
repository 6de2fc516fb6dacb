"""Parity of the CUDA engine with the CPU oracle (bit-exact, integer counts).

Each case builds the graph on the GPU through the C ABI (kcgpu_b200 -> libkc.so)
and compares with oracle/oracle.cpp on the same seeded edge list.
"""
import math

import numpy as np
import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph
from tests import graphs as G

pytestmark = pytest.mark.gpu

VARIANTS = [(mode, unit, enc) for mode in ("orient", "pivot", "auto") for unit in ("node", "edge")
            for enc in ("bitmap", "list")]


def _seeded_graphs():
    out = []
    for seed, (n, p) in enumerate([(60, 0.3), (300, 0.08), (2000, 0.01), (800, 0.05)]):
        s, d, nn = kc.gen_er(n, p, 100 + seed).arrays()
        out.append((f"er{n}", s, d, nn))
    s, d, nn = kc.gen_sbm(400, 4, 0.3, 0.02, 7).arrays()
    out.append(("sbm400", s, d, nn))
    el = kc.gen_er(500, 0.02, 11)
    el.plant_cliques(3, 12, 18, 3)
    s, d, nn = el.arrays()
    out.append(("planted500", s, d, nn))
    s, d, nn = kc.gen_rmat(11, 8, seed=5).arrays()
    out.append(("rmat11", s, d, nn))
    s, d, nn = kc.gen_chung_lu(3000, 2.1, 10, 300, 9).arrays()
    out.append(("chunglu3k", s, d, nn))
    return out


GRAPHS = None


def graphs():
    global GRAPHS
    if GRAPHS is None:
        GRAPHS = _seeded_graphs()
    return GRAPHS


@pytest.mark.parametrize("gi", range(8))
@pytest.mark.parametrize("orientation", ["degree", "degen"])
def test_counts_match_oracle(ctx, gi, orientation):
    name, s, d, n = graphs()[gi]
    og = OracleGraph(s, d, n)
    og.orient(orientation)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient(orientation)
        for k in (3, 4, 5, 6, 7):
            want = og.count(k, "pivot")
            for mode, unit, enc in VARIANTS:
                for part in (1, 8, 32):
                    got = g.count(k, mode=mode, unit=unit, part=part, encoding=enc)
                    assert got == want, f"{name} {orientation} k={k} {mode}/{unit}/{enc}/p{part}: {got} != {want}"


@pytest.mark.parametrize("orientation", ["degree", "degen"])
def test_csr_dag_and_peel_match_oracle(ctx, orientation):
    for name, s, d, n in graphs():
        ms, md = G.messy(s, d, n, 3)
        og = OracleGraph(ms, md, n)
        og.orient(orientation)
        with kc.Graph.from_edges(ctx, ms, md, n) as g:
            rp, ci = g.csr()
            orp, oci = og.csr()
            assert np.array_equal(rp, orp) and np.array_equal(ci, oci), name
            g.orient(orientation)
            rp, ci = g.dag()
            orp, oci = og.dag()
            assert np.array_equal(rp, orp) and np.array_equal(ci, oci), f"{name} dag"
            if orientation == "degen":
                prio, lev = g.peel()
                oprio, olev = og.peel()
                assert np.array_equal(lev, olev), f"{name} peel level"
                assert np.array_equal(prio, oprio), f"{name} peel priority"


def test_kcore_and_truss_support(ctx):
    for name, s, d, n in graphs():
        og = OracleGraph(s, d, n)
        with kc.Graph.from_edges(ctx, s, d, n) as g:
            core, mx = g.kcore()
            ocore, omx = og.kcore()
            assert mx == omx and np.array_equal(core, ocore), name
            assert np.array_equal(g.truss_support(), og.truss_support()), name


def test_known_answers_complete_graphs(ctx):
    for n in (1, 2, 3, 8, 31, 32, 33, 64, 65):
        s, d = G.complete(n)
        with kc.Graph.from_edges(ctx, s, d, n) as g:
            g.orient("degen")
            for k in range(1, min(n, 9) + 2):
                for mode, unit, enc in VARIANTS:
                    if unit == "edge" and k == 1:
                        continue
                    if mode == "orient" and math.comb(n, k) > 5e7:
                        continue
                    assert g.count(k, mode=mode, unit=unit, encoding=enc) == math.comb(n, k), (n, k, mode, unit, enc)


def test_u128_counts(ctx):
    # C(130, 65) ~ 9.5e37 needs the high word
    n = 130
    s, d = G.complete(n)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        for k in (40, 65, 90, 130):
            for unit in ("node", "edge"):
                got = g.count(k, mode="pivot", unit=unit, encoding="bitmap")
                assert got == math.comb(n, k), (k, unit)
        assert g.count(65, mode="pivot", unit="node", encoding="list") == math.comb(n, 65)


def test_edgeless_union_multipartite(ctx):
    # edgeless
    with kc.Graph.from_edges(ctx, np.zeros(0, np.uint32), np.zeros(0, np.uint32), 10) as g:
        g.orient("degree")
        assert g.count(1) == 10 and g.count(2) == 0 and g.count(3) == 0
        assert g.count(3, mode="pivot", unit="edge") == 0
    # disjoint union is additive
    parts = [G.complete(7) + (7,), G.complete(12) + (12,), tuple(kc.gen_er(200, 0.1, 4).arrays())]
    s, d, n = G.disjoint_union(parts)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        for k in (3, 4, 5):
            total = 0
            for ps, pd, pn in parts:
                with kc.Graph.from_edges(ctx, ps, pd, pn) as h:
                    h.orient("degen")
                    total += h.count(k, mode="pivot")
            for mode, unit, enc in VARIANTS:
                assert g.count(k, mode=mode, unit=unit, encoding=enc) == total
    # complete multipartite graphs: e_k(part sizes)
    for sizes in ([3, 3, 3], [5, 1, 4, 2], [10, 10, 10, 10, 10], [2] * 12):
        s, d, n = G.multipartite(sizes)
        with kc.Graph.from_edges(ctx, s, d, n) as g:
            g.orient("degree")
            for k in range(3, len(sizes) + 2):
                want = G.multipartite_kcliques(sizes, k)
                for mode, unit, enc in VARIANTS:
                    assert g.count(k, mode=mode, unit=unit, encoding=enc) == want, (sizes, k, mode, unit, enc)


def test_heavy_units_handed_on(ctx):
    # planted cliques of 28-32 vertices: the lowest clique vertex's unit needs
    # far more traversal nodes than a warp unit's budget, so it is counted
    # again by the CTA-wide heavy pass; the count must not change.
    el = kc.gen_er(400, 0.04, 31)
    el.plant_cliques(2, 28, 32, 8)
    s, d, n = el.arrays()
    og = OracleGraph(s, d, n)
    og.orient("degree")
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        for k in (5, 7, 9):
            want = og.count(k, "pivot")
            for mode in ("orient", "pivot", "auto"):
                for unit in ("node", "edge"):
                    for part in (0, 4, 32):
                        got = g.count(k, mode=mode, unit=unit, part=part)
                        assert got == want, (k, mode, unit, part)


def test_batched_matches_single_graph_counts(ctx):
    e = kc.gen_batch(60, 77)
    s, d, _ = e.arrays()
    off, nn, kk, fam = e.batch_meta()
    for orientation in ("degree", "degen"):
        counts, choice, st = kc.batch_count(ctx, s, d, off, nn, kk, orientation=orientation, return_choice=True,
                                            return_stats=True)
        assert st["n_graphs"] == 60 and st["tree_nodes"] > 0
        for g in range(60):
            a, b = int(off[g]), int(off[g + 1])
            og = OracleGraph(s[a:b], d[a:b], int(nn[g]))
            og.orient(orientation)
            assert counts[g] == og.count(int(kk[g]), "pivot"), (orientation, g, choice[g])


def test_relabel_invariance(ctx):
    s, d, n = kc.gen_sbm(600, 4, 0.2, 0.01, 21).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        base = [g.count(k, mode="pivot") for k in (3, 4, 5)]
    ps, pd = G.relabel(s, d, n, 99)
    with kc.Graph.from_edges(ctx, ps, pd, n) as g:
        g.orient("degen")
        assert [g.count(k, mode="orient") for k in (3, 4, 5)] == base


def test_determinism(ctx):
    s, d, n = kc.gen_rmat(12, 8, seed=3).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        a = [g.count(5, mode=m, unit=u) for m in ("orient", "pivot") for u in ("node", "edge")]
        b = [g.count(5, mode=m, unit=u) for m in ("orient", "pivot") for u in ("node", "edge")]
        assert a == b and len(set(a)) == 1


def test_errors(ctx):
    s, d = G.complete(5)
    with kc.Graph.from_edges(ctx, s, d, 5) as g:
        with pytest.raises(kc.KCError) as e:
            g.count(3)
        assert e.value.name == "KC_ERR_NOT_ORIENTED"
        g.orient("degree")
        with pytest.raises(kc.KCError) as e:
            g.count(0)
        assert e.value.name == "KC_ERR_INVALID_ARG"
        with pytest.raises(kc.KCError) as e:
            g.count(3, part=3)
        assert e.value.name == "KC_ERR_INVALID_ARG"
        with pytest.raises(kc.KCError):
            g.orient(7)
    with pytest.raises(kc.KCError) as e:
        kc.Graph.from_edges(ctx, np.array([0, 9], np.uint32), np.array([1, 2], np.uint32), 5)
    assert e.value.name == "KC_ERR_INVALID_ARG"


def test_reference_driver_mirror(ctx):
    s, d, n = kc.gen_er(1000, 0.03, 2).arrays()
    og = OracleGraph(s, d, n)
    og.orient("degree")
    want = og.count(5)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        mc = kc.SingleGPU_Kclique(0, g)
        for name in ("node_async", "node_binary_async", "node_pivot_async", "node_nobin_pivot_async",
                     "edge_async", "edge_binary_async", "edge_pivot_async", "edge_nobin_pivot_async"):
            for part in (1, 2, 4, 8, 16, 32):
                assert getattr(mc, "findKclqueIncremental_" + name)(5, part) == want
                assert mc.count() == want


def test_stats_flag(ctx):
    s, d, n = kc.gen_er(2000, 0.01, 1).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        r = g.count(4, stats=True)
        assert r.stats["units"] > 0 and r.stats["tree_nodes"] > 0 and r.stats["ms_total"] > 0


def test_units_above_1024_vertices(ctx):
    # Complete tripartite K(600, 600, 600) under degree orientation (all
    # degrees equal, ties by id): the first vertices have out-degree up to
    # 1200, so their units take the launch whose bitmap and frames live in
    # global memory. Closed form: 600^3 triangles, no 4-cliques.
    sizes = [600, 600, 600]
    s, d, n = G.multipartite(sizes)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        assert g.info()["max_out_degree"] > 1024
        for k in (3, 4):
            want = G.multipartite_kcliques(sizes, k)
            for mode, unit, enc in VARIANTS:
                assert g.count(k, mode=mode, unit=unit, encoding=enc) == want, (k, mode, unit, enc)


def test_pivot_cta_units_with_tail_helping(ctx):
    """Four dense blocks (p 0.5, 350 vertices each): a few dozen units above
    128 vertices, counted by a CTA each with pivoting, far fewer than the
    launch's CTAs, so most CTAs join units still being walked (tail helping)
    and take cut nodes by the unit's global ticket. Every count equals the
    oracle's, in every pivoting variant and partition size."""
    s, d, n = kc.gen_sbm(1400, 4, 0.5, 0.001, 7).arrays()
    og = OracleGraph(s, d, n)
    assert og.orient("degen") > 128
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        for k in (6, 9):
            want = og.count(k, "pivot", closed=True)
            for mode in ("pivot", "auto"):
                for unit in ("node", "edge"):
                    for part in (4, 32):
                        assert g.count(k, mode=mode, unit=unit, part=part) == want, (k, mode, unit, part)
            # repeated counts agree (helpers join at different moments each time)
            assert [g.count(k, mode="pivot", unit="node", part=32) for _ in range(3)] == [want] * 3
