"""Several k in one pivoting walk (kc_count_multi): every count equals the
single-k count and the CPU oracle's, for node and edge units, k sets that
include k <= 2, the unit-level closed forms (k = held + 1, + 2) and k far
above the clique number, in any order and with repeats."""
import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph

pytestmark = pytest.mark.gpu


def _graphs():
    out = []
    s, d, n = kc.gen_rmat(12, 12, 0.57, 0.19, 0.19, seed=8).arrays()
    out.append(("rmat12", s, d, n))
    el = kc.gen_er(1500, 0.01, 31)
    el.plant_cliques(3, 14, 24, 2)
    s, d, n = el.arrays()
    out.append(("planted1500", s, d, n))
    s, d, n = kc.gen_sbm(1400, 4, 0.5, 0.001, 7).arrays()  # units above 128 vertices
    out.append(("sbm_dense", s, d, n))
    return out


@pytest.mark.parametrize("gi", [0, 1, 2])
def test_multi_k_equals_single_k_and_oracle(ctx, gi):
    name, s, d, n = _graphs()[gi]
    og = OracleGraph(s, d, n)
    og.orient("degen")
    ks = [3, 4, 5, 6, 7, 9, 12, 15, 30]
    want = {k: og.count(k, "pivot", closed=True) for k in ks}
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        info = g.info()
        want[1], want[2] = info["n"], info["m"]
        for unit in ("node", "edge"):
            got = g.count_multi(ks, unit=unit)
            assert got == [want[k] for k in ks], (name, unit)
            assert g.count_multi([2, 1] + ks[::-1] + [5, 5], unit=unit) == \
                [want[2], want[1]] + [want[k] for k in ks[::-1]] + [want[5]] * 2, (name, unit)
        for k in (4, 6):  # one k through the several-k walk equals kc_count
            assert g.count_multi([k]) == [g.count(k, mode="pivot", unit="node", part=32)]


def test_multi_k_arguments(ctx):
    s, d, n = kc.gen_er(200, 0.05, 3).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        with pytest.raises(kc.KCError) as e:
            g.count_multi([3, 4])
        assert e.value.name == "KC_ERR_NOT_ORIENTED"
        g.orient("degree")
        for bad in ([], list(range(3, 36)), [0, 3]):
            with pytest.raises(kc.KCError) as e:
                g.count_multi(bad)
            assert e.value.name == "KC_ERR_INVALID_ARG"
