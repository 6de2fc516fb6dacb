"""Local (per-vertex) clique counts, the reference's -m lkc: bit-exact against
the oracle's listing, closed forms, and the global counts."""
import math

import numpy as np
import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph
from tests import graphs as G

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    for seed, (n, p) in enumerate([(60, 0.3), (300, 0.08), (800, 0.05)]):
        out.append((f"er{n}",) + tuple(kc.gen_er(n, p, 100 + seed).arrays()))
    out.append(("sbm400",) + tuple(kc.gen_sbm(400, 4, 0.3, 0.02, 7).arrays()))
    el = kc.gen_er(500, 0.02, 11)
    el.plant_cliques(3, 12, 18, 3)
    out.append(("planted500",) + tuple(el.arrays()))
    out.append(("rmat11",) + tuple(kc.gen_rmat(11, 8, seed=5).arrays()))
    return out


@pytest.mark.parametrize("orientation", ["degree", "degen"])
def test_local_counts_match_oracle(ctx, orientation):
    for name, s, d, n in _cases():
        og = OracleGraph(s, d, n)
        og.orient(orientation)
        with kc.Graph.from_edges(ctx, s, d, n) as g:
            g.orient(orientation)
            for k in (1, 2, 3, 4, 5, 7, 9):
                want = og.count_local(k)
                for mode, unit, part in (("orient", "node", 0), ("orient", "node", 8), ("orient", "edge", 1),
                                         ("orient", "edge", 32), ("pivot", "node", 0), ("pivot", "node", 8),
                                         ("pivot", "edge", 0), ("pivot", "edge", 2), ("auto", "node", 0),
                                         ("auto", "edge", 0)):
                    got = g.count_local(k, unit=unit, part=part, mode=mode)
                    assert got == want, (name, orientation, k, mode, unit, part)
                assert sum(want) == k * g.count(k, mode="pivot")


def test_local_counts_closed_forms(ctx):
    n = 40
    s, d = G.complete(n)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        for k in (3, 6, 9):
            for unit in ("node", "edge"):
                assert g.count_local(k, unit=unit) == [math.comb(n - 1, k - 1)] * n
        for k in (12, 20, 40):  # pivoting: counts well past 2^64 per vertex at n = 130 below
            assert g.count_local(k, mode="pivot") == [math.comb(n - 1, k - 1)] * n
    n = 130
    s, d = G.complete(n)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        for unit in ("node", "edge"):
            assert g.count_local(66, unit=unit, mode="pivot") == [math.comb(n - 1, 65)] * n
    # K(600, 600, 600): units above 1024 vertices; every vertex is in 600^2
    # triangles and no 4-clique
    sizes = [600, 600, 600]
    s, d, n = G.multipartite(sizes)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        for unit in ("node", "edge"):
            for mode in ("orient", "pivot"):
                assert g.count_local(3, unit=unit, mode=mode) == [600 * 600] * n
                assert g.count_local(4, unit=unit, mode=mode) == [0] * n


def test_local_counts_reference_mirror_and_errors(ctx):
    s, d, n = kc.gen_er(200, 0.1, 3).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        ref = kc.SingleGPU_Kclique_Local(0, g)
        a = ref.findKclqueIncremental_node_binary_async_local(4, 8)
        b = ref.findKclqueIncremental_edge_binary_async_local(4, 8)
        c = ref.findKclqueIncremental_node_pivot_async_local(4, 8)
        e = ref.findKclqueIncremental_edge_pivot_async_local(4, 8)
        assert a == b == c == e and sum(a) == 4 * g.count(4)
        p = kc._lib.KcParams()
        p.k, p.mode, p.unit, p.part, p.encoding = 4, 0, 0, 8, 1  # list encoding: not supported
        out = (kc._lib.KcU128 * n)()
        assert kc.lib().kc_count_local(g._h, kc.C.byref(p), out, None) != 0
