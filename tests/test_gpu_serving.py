"""The request server: results are exact whether a request runs alone or in a
mix of concurrent requests; cancellation and HBM admission behave."""
import numpy as np
import pytest

import kcgpu_b200 as kc

pytestmark = pytest.mark.gpu


def _alone(ctx, s, d, n, k, orientation="degen"):
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient(orientation)
        return g.count(k, mode="pivot")


def test_mixed_requests_match_lone_counts(ctx):
    graphs = [kc.gen_rmat(sc, 8, seed=sc).arrays() for sc in (9, 10, 11, 12)]
    graphs.append(kc.gen_er(1500, 0.02, 3).arrays())
    el = kc.gen_er(300, 0.03, 5)
    el.plant_cliques(1, 25, 25, 2)
    graphs.append(el.arrays())
    rng = np.random.default_rng(0)
    with kc.Server(ctx, streams=4) as srv:
        ids = [srv.put_graph(s, d, n) for s, d, n in graphs]
        jobs = []
        for i in range(48):
            gi = int(rng.integers(len(graphs)))
            k = int(rng.integers(3, 9))
            if i % 3 == 0:  # one-shot requests carry their own edge list
                s, d, n = graphs[gi]
                jobs.append((srv.submit_edges(s, d, n, k), gi, k))
            else:
                jobs.append((srv.submit(ids[gi], k), gi, k))
        want = {}
        for t, gi, k in jobs:
            r = srv.wait(t)
            if (gi, k) not in want:
                want[(gi, k)] = _alone(ctx, *graphs[gi], k)
            assert r["count"] == want[(gi, k)], (gi, k)
            assert r["submit_ms"] <= r["start_ms"] <= r["done_ms"]


def test_requests_overlap_on_the_device(ctx):
    # four resident graphs (each owned by another worker context) and eight
    # requests: a later request starts while an earlier one is still running
    graphs = [kc.gen_rmat(14, 16, seed=30 + i).arrays() for i in range(4)]
    with kc.Server(ctx, streams=4) as srv:
        ids = [srv.put_graph(s, d, n) for s, d, n in graphs]
        tickets = [(srv.submit(ids[i % 4], 7), i % 4) for i in range(8)]
        res = [(srv.wait(t), gi) for t, gi in tickets]
    overlapped = any(b["start_ms"] < a["done_ms"] and a["start_ms"] <= b["start_ms"]
                     for i, (a, _) in enumerate(res) for (b, _) in res[i + 1:])
    assert overlapped, [(r["start_ms"], r["done_ms"]) for r, _ in res]
    want = {gi: _alone(ctx, *graphs[gi], 7) for gi in range(4)}
    for r, gi in res:
        assert r["count"] == want[gi]


def test_admission_passes_a_blocked_head(ctx):
    # The budget holds the large request A and a small one, not two large
    # ones: B (large, behind A) must wait, C (small, behind B) passes it.
    big = kc.gen_rmat(15, 16, seed=7).arrays()
    small = kc.gen_er(400, 0.05, 8).arrays()
    fp_big = kc.footprint_bytes(big[2], len(big[0]), 0)
    fp_small = kc.footprint_bytes(small[2], len(small[0]), 0)
    budget = fp_big + fp_small + (fp_big - fp_small) // 2
    with kc.Server(ctx, hbm_budget_bytes=budget, streams=4) as srv:
        ta = srv.submit_edges(*big, 8)
        tb = srv.submit_edges(*big, 8)
        tc = srv.submit_edges(*small, 4)
        a, b, c = srv.wait(ta), srv.wait(tb), srv.wait(tc)
    assert c["start_ms"] < b["start_ms"]
    assert b["start_ms"] >= a["done_ms"]  # never two large requests on the device at once
    assert a["count"] == b["count"] == _alone(ctx, *big, 8)
    assert c["count"] == _alone(ctx, *small, 4)


def test_cancel_and_admission(ctx):
    s, d, n = kc.gen_rmat(13, 16, seed=1).arrays()
    bs, bd, bn = kc.gen_rmat(15, 10, seed=2).arrays()
    with kc.Server(ctx, streams=1) as srv:
        gid = srv.put_graph(s, d, n)
        # a long one-shot request holds the one worker; requests for the
        # resident graph queue behind it (and later run as one walk)
        busy = srv.submit_edges(bs, bd, bn, 12)
        tickets = [srv.submit(gid, 6) for _ in range(6)]
        srv.cancel(tickets[-1])  # still queued
        with pytest.raises(kc.KCError) as e:
            srv.wait(tickets[-1])
        assert e.value.name == "KC_ERR_CANCELLED"
        counts = {srv.wait(t)["count"] for t in tickets[:-1]}
        assert counts == {_alone(ctx, s, d, n, 6)}
        assert srv.wait(busy)["count"] == _alone(ctx, bs, bd, bn, 12)
    # a budget smaller than one graph's projected footprint is rejected up front
    with kc.Server(ctx, hbm_budget_bytes=1 << 20, streams=1) as srv:
        with pytest.raises(kc.KCError) as e:
            srv.put_graph(s, d, n)
        assert e.value.name == "KC_ERR_ADMISSION"
        with pytest.raises(kc.KCError) as e:
            srv.submit_edges(s, d, n, 4)
        assert e.value.name == "KC_ERR_ADMISSION"


def test_queued_requests_of_a_resident_graph_share_one_walk(ctx):
    """Requests for one resident graph that queue together run as one walk
    for all their k (the same start and end), each with its own exact count."""
    s, d, n = kc.gen_rmat(12, 12, seed=4).arrays()
    bs, bd, bn = kc.gen_rmat(15, 10, seed=2).arrays()
    ks = [3, 5, 7, 7, 9, 12, 15]
    with kc.Server(ctx, streams=1) as srv:
        gid = srv.put_graph(s, d, n)
        busy = srv.submit_edges(bs, bd, bn, 12)  # holds the one worker meanwhile
        tickets = [srv.submit(gid, k) for k in ks]
        res = [srv.wait(t) for t in tickets]
        srv.wait(busy)
    # taken from the queue together (within a millisecond) and done together
    assert len({r["done_ms"] for r in res}) == 1
    assert max(r["start_ms"] for r in res) - min(r["start_ms"] for r in res) < 1.0
    for k, r in zip(ks, res):
        assert r["count"] == _alone(ctx, s, d, n, k), k
