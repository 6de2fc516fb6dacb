"""Unit shards (kc_count_shard): the shards of a count, run one after another
on one GPU, add up to the whole count, which equals the CPU oracle's, in
every mode, unit and encoding and for shard counts that do and do not divide
the class sizes; every unit is counted by exactly one shard."""
import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph

pytestmark = pytest.mark.gpu

VARIANTS = [("orient", "node", "bitmap"), ("orient", "edge", "list"), ("pivot", "node", "bitmap"),
            ("pivot", "edge", "bitmap"), ("pivot", "node", "list"), ("auto", "node", "bitmap")]


def _graphs():
    out = []
    s, d, n = kc.gen_rmat(13, 16, 0.57, 0.19, 0.19, seed=4).arrays()
    out.append(("rmat13", s, d, n))
    el = kc.gen_er(3000, 0.01, 21)
    el.plant_cliques(4, 25, 40, 5)
    s, d, n = el.arrays()
    out.append(("planted3k", s, d, n))
    return out


@pytest.mark.parametrize("gi", [0, 1])
def test_shards_add_up_to_the_count(ctx, gi):
    name, s, d, n = _graphs()[gi]
    og = OracleGraph(s, d, n)
    og.orient("degen")
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        for k in (4, 6):
            want = og.count(k, "pivot", closed=True)
            for mode, unit, enc in VARIANTS:
                whole = g.count(k, mode=mode, unit=unit, part=8, encoding=enc, stats=True)
                assert whole.count == want, (name, k, mode, unit, enc)
                for S in (2, 3, 8):
                    parts = [g.count(k, mode=mode, unit=unit, part=8, encoding=enc, stats=True, shard=(i, S))
                             for i in range(S)]
                    assert sum(r.count for r in parts) == want, (name, k, mode, unit, enc, S)
                    # each unit in exactly one shard
                    assert sum(r.stats["units"] for r in parts) == whole.stats["units"], (name, k, mode, S)


def test_shard_arguments_and_small_k(ctx):
    s, d, n = kc.gen_er(200, 0.05, 3).arrays()
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        info = g.info()
        # k <= 2 needs no units: shard 0 holds the whole count
        assert [g.count(1, shard=(i, 3)) for i in range(3)] == [info["n"], 0, 0]
        assert [g.count(2, shard=(i, 3)) for i in range(3)] == [info["m"], 0, 0]
        # more shards than units: the empty shards count 0 and the sum holds
        whole = g.count(3, mode="orient", unit="node", part=8)
        many = [g.count(3, mode="orient", unit="node", part=8, shard=(i, 257)) for i in range(257)]
        assert sum(many) == whole and many.count(0) >= 257 - info["n"]
        for bad in ((3, 3), (0, 0)):
            with pytest.raises(kc.KCError) as e:
                g.count(3, shard=bad)
            assert e.value.name == "KC_ERR_INVALID_ARG"
