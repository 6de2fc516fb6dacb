"""Host-input batches counted as a pipeline of chunks (the next chunk's
host->device copy overlapping the current chunk's build and count): the
counts and choices equal the one-pass call's, for chunk sizes from one graph
per chunk to the whole batch, and the statistics add up over the chunks."""
import numpy as np
import pytest

import kcgpu_b200 as kc

pytestmark = pytest.mark.gpu

NEVER = 2**64 - 1


def _batch():
    el = kc.gen_batch(40, 77, n_max=1500)
    s, d, _ = el.arrays()
    off, nn, kk, _ = el.batch_meta()
    return s, d, off, nn, kk


def test_chunked_batches_match_one_pass(ctx):
    s, d, off, nn, kk = _batch()
    try:
        ctx.set_batch_chunk_edges(NEVER)
        want, wchoice, wst = kc.batch_count(ctx, s, d, off, nn, kk, return_choice=True, return_stats=True)
        E = int(off[-1])
        for chunk in (1, 5000, E // 3, E - 1):
            ctx.set_batch_chunk_edges(chunk)
            got, choice, st = kc.batch_count(ctx, s, d, off, nn, kk, return_choice=True, return_stats=True)
            assert got == want, chunk
            assert choice == wchoice, chunk
            assert st["n_graphs"] == len(nn)
            assert st["units"] == wst["units"] and st["n_vertices"] == wst["n_vertices"], chunk
            assert st["ms_h2d"] > 0
    finally:
        ctx.set_batch_chunk_edges(0)


def test_chunked_batch_reports_bad_graph(ctx):
    s, d, off, nn, kk = _batch()
    kk = np.array(kk, copy=True)
    kk[len(kk) - 3] = 0  # a graph in the last chunk asks for k = 0
    try:
        ctx.set_batch_chunk_edges(5000)
        with pytest.raises(kc.KCError) as e:
            kc.batch_count(ctx, s, d, off, nn, kk)
        assert e.value.name == "KC_ERR_INVALID_ARG"
        ctx.set_batch_chunk_edges(NEVER)
        kk[len(kk) - 3] = 4
        assert kc.batch_count(ctx, s, d, off, nn, kk)  # the context is still usable
    finally:
        ctx.set_batch_chunk_edges(0)


def test_per_graph_methods_given_by_the_caller(ctx):
    """kc_batch_opts.graph_params: every graph on the method the caller names
    (several passes side by side, in one pass and as a pipeline); the counts
    equal the autotuned batch's and each graph reports its method."""
    s, d, off, nn, kk = _batch()
    methods = [{"mode": "pivot", "unit": "node", "part": 8, "encoding": "bitmap"},
               {"mode": "orient", "unit": "edge", "part": 4, "encoding": "bitmap"},
               {"mode": "auto", "unit": "node", "part": 32, "encoding": "list"},
               {"mode": "pivot", "unit": "edge", "part": 0, "encoding": "list"}]
    gp = [methods[i % len(methods)] for i in range(len(nn))]
    try:
        ctx.set_batch_chunk_edges(NEVER)
        want = kc.batch_count(ctx, s, d, off, nn, kk)
        for chunk in (NEVER, 5000):
            ctx.set_batch_chunk_edges(chunk)
            got, choice = kc.batch_count(ctx, s, d, off, nn, kk, graph_params=gp, return_choice=True)
            assert got == want, chunk
            for i, c in enumerate(choice):
                m = gp[i]
                if int(kk[i]) > 2:
                    assert (c["mode"], c["unit"], c["part"], c["encoding"]) == (
                        kc.MODES[m["mode"]], kc.UNITS[m["unit"]], m["part"], kc.ENCODINGS[m["encoding"]]), i
    finally:
        ctx.set_batch_chunk_edges(0)
