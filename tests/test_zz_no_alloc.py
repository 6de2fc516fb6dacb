"""kc_truss_support_noalloc: the allocation-free truss-support entry point.

Some callers cannot allocate device memory while they run (a plugin inside a
host runtime that owns the GPU's memory, a latency-critical stream that must
not be stalled by cudaMalloc/cudaFree, a pipeline that reserves everything up
front). This entry point serves them with caller-provided device buffers and a
fixed scratch array compiled into the library. The test calls it through the C
ABI twice in a row, on two different graphs so a stale scratch would show, and
compares each result with the allocating entry point kc_truss_support (exact
integers: the tolerance is zero).

The file name sorts last so a run that stops at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import kcgpu_b200 as kc

pytestmark = pytest.mark.gpu


def _noalloc_support(ctx, g):
    import torch

    rp, ci = g.csr()
    m = g.m
    d_rp = torch.from_numpy(rp.view(np.int32)).cuda()
    d_ci = torch.from_numpy(ci.view(np.int32) if ci.size else np.zeros(1, np.int32)).cuda()
    d_sup = torch.full((max(1, m),), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = kc.lib().kc_truss_support_noalloc(C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_ci.data_ptr()), rp.size - 1,
                                          C.c_void_p(d_sup.data_ptr()), C.c_void_p(stream.cuda_stream))
    kc.check(st)
    stream.synchronize()
    return d_sup[:m].cpu().numpy().view(np.uint32)


def test_noalloc_truss_support_matches_allocating_entry_point():
    from oracle.oracle import OracleGraph

    ctx = kc.Context(0)
    try:
        first = kc.gen_er(3000, 0.01, 17).arrays()
        second = kc.gen_rmat(10, 8, seed=4).arrays()
        at_limit = kc.gen_er(1 << 18, 1e-5, 23).arrays()  # n_nodes at the array's limit, sparse
        no_edges = (np.zeros(0, np.uint32), np.zeros(0, np.uint32), 5)
        for s, d, n in (first, second, at_limit, no_edges):
            with kc.Graph.from_edges(ctx, s, d, n) as g:
                assert g.info()["n"] == n
                want = g.truss_support()
                got = _noalloc_support(ctx, g)
                assert got.shape == want.shape
                assert np.array_equal(got, want)
                assert np.array_equal(got, OracleGraph(s, d, n).truss_support())
    finally:
        ctx.close()


def test_noalloc_rejects_graphs_above_its_limit():
    st = kc.lib().kc_truss_support_noalloc(C.c_void_p(1), C.c_void_p(1), (1 << 18) + 1, C.c_void_p(1), None)
    assert st == 1  # KC_ERR_INVALID_ARG, nothing launched
    assert b"at most 262144" in kc.lib().kc_last_error()
