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


def test_cancel_and_admission(ctx):
    s, d, n = kc.gen_rmat(13, 16, seed=1).arrays()
    with kc.Server(ctx, streams=1) as srv:
        gid = srv.put_graph(s, d, n)
        tickets = [srv.submit(gid, 6) for _ in range(6)]
        srv.cancel(tickets[-1])  # still queued behind the others on one slot
        with pytest.raises(kc.KCError) as e:
            srv.wait(tickets[-1])
        assert e.value.name == "KC_ERR_CANCELLED"
        counts = {srv.wait(t)["count"] for t in tickets[:-1]}
        assert counts == {_alone(ctx, s, d, n, 6)}
    # a budget smaller than one graph's projected footprint is rejected up front
    with kc.Server(ctx, hbm_budget_bytes=1 << 20, streams=1) as srv:
        with pytest.raises(kc.KCError) as e:
            srv.put_graph(s, d, n)
        assert e.value.name == "KC_ERR_ADMISSION"
        with pytest.raises(kc.KCError) as e:
            srv.submit_edges(s, d, n, 4)
        assert e.value.name == "KC_ERR_ADMISSION"
