"""Failure paths, driven from the host: no GPU fault, trap or hang.

* The device time limit (kc_ctx_set_time_limit): the counting kernels read the
  GPU's global timer when a unit group takes its next unit and stop taking
  units past the limit; the call returns KC_ERR_DEVICE_TIMEOUT and the context
  counts correctly afterwards.
* Allocation failure (kc_test_fail_alloc_after): every device allocation the
  library makes (single graphs, batches in one pass and as a pipeline of
  chunks) is made to fail in turn; each failing call must return
  KC_ERR_OOM and leave no device allocation behind
  (kc_test_live_allocations), and the calls succeed again once the injection
  stops.
"""
import numpy as np
import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph

pytestmark = pytest.mark.gpu


def test_time_limit_stops_counting_and_context_recovers(ctx):
    s, d, n = kc.gen_rmat(14, 16, 0.57, 0.19, 0.19, seed=3).arrays()
    og = OracleGraph(s, d, n)
    og.orient("degen")
    want = og.count(5, "pivot", closed=True)
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        ctx.set_time_limit(1)
        try:
            for mode, unit, enc in (("pivot", "node", "bitmap"), ("orient", "node", "bitmap"),
                                    ("pivot", "edge", "list"), ("auto", "node", "bitmap")):
                with pytest.raises(kc.KCError) as e:
                    g.count(5, mode=mode, unit=unit, part=8, encoding=enc)
                assert e.value.name == "KC_ERR_DEVICE_TIMEOUT", (mode, unit, enc)
            el = kc.gen_batch(20, 5)
            bs, bd, _ = el.arrays()
            off, nn, kk, _ = el.batch_meta()
            with pytest.raises(kc.KCError) as e:
                kc.batch_count(ctx, bs, bd, off, nn, kk)
            assert e.value.name == "KC_ERR_DEVICE_TIMEOUT"
        finally:
            ctx.set_time_limit(0)
        assert g.count(5, mode="pivot", unit="node", part=8) == want
        assert g.count(5, mode="orient", unit="edge", part=8) == want
        ctx.set_time_limit(60 * 10**9)  # a generous limit does not get in the way
        try:
            assert g.count(5, mode="auto", unit="node", part=0) == want
        finally:
            ctx.set_time_limit(0)


def _every_entry_point(ctx, s, d, n, bs, bd, off, nn, kk):
    out = []
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degen")
        for mode in ("orient", "pivot", "auto"):
            for unit in ("node", "edge"):
                for enc in ("bitmap", "list"):
                    out.append(g.count(5, mode=mode, unit=unit, part=8, encoding=enc))
        out.append(tuple(g.kcore()[0].tolist()))
        out.append(tuple(g.truss_support().tolist()))
        out.append(tuple(g.count_local(4)))
    with kc.Graph.from_edges(ctx, s, d, n) as g:
        g.orient("degree")
        out.append(g.count(4, mode="pivot", unit="edge", part=4))
    out.append(tuple(kc.batch_count(ctx, bs, bd, off, nn, kk)))
    ctx.set_batch_chunk_edges(2000)  # the same batch as a pipeline of chunks
    try:
        out.append(tuple(kc.batch_count(ctx, bs, bd, off, nn, kk)))
    finally:
        ctx.set_batch_chunk_edges(0)
    return out


def test_allocation_failures_return_oom_and_leak_nothing(ctx):
    L = kc.lib()
    s, d, n = kc.gen_er(300, 0.08, 5).plant_cliques(1, 12, 12, 3).arrays()
    el = kc.gen_batch(12, 9, n_max=400)
    bs, bd, _ = el.arrays()
    off, nn, kk, _ = el.batch_meta()
    want = _every_entry_point(ctx, s, d, n, bs, bd, off, nn, kk)  # also sizes the binomial table
    # the context's block cache would serve repeated allocations without the
    # driver: empty it, so that every allocation of the sequence is a real one
    L.kc_ctx_release_cached_memory(ctx.handle)
    base = L.kc_test_live_allocations()
    failures = 0
    for i in range(5000):
        L.kc_ctx_release_cached_memory(ctx.handle)
        L.kc_test_fail_alloc_after(i)
        try:
            got = _every_entry_point(ctx, s, d, n, bs, bd, off, nn, kk)
            failed = False
        except kc.KCError as e:
            assert e.name == "KC_ERR_OOM", (i, str(e))
            failed = True
        finally:
            L.kc_test_fail_alloc_after(-1)
        L.kc_ctx_release_cached_memory(ctx.handle)
        assert L.kc_test_live_allocations() == base, f"allocation {i} failed: {L.kc_test_live_allocations() - base} left"
        if not failed:
            assert got == want
            break
        failures += 1
    else:
        pytest.fail("the injection never ran out of allocations")
    # every real allocation of the sequence was made to fail once (the block
    # cache serves the repeated ones within the sequence)
    assert failures > 20
