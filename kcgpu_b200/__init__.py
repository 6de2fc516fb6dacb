"""kcgpu_b200 — exact k-clique counting on one B200.

Python front end of libkc.so (C ABI: include/kc.h). Every call runs the CUDA
engine; nothing here computes a count on the CPU.

Mirrors the `-m kc` path of KCGPU:
  * ``Graph.from_edges`` / ``Graph.from_csr``  ~ EdgeListFile + CSRCOO::from_edgelist
    (include/FIleReader.cuh:383-411, include/CSRCOO.cuh:37-80), built on the GPU;
  * ``Graph.orient("degree"|"degen")``         ~ src/main.cu:164-229;
  * ``Graph.count(k, mode, unit, part, encoding)`` and the
    ``SingleGPU_Kclique`` class below            ~ kclique/kclique.cuh:1302-2643;
  * ``parse_spec("o8b")``                       ~ parseKcConfig, include/Config.h:235-271.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import KCError, KcBatchOpts, KcBatchStats, KcCountStats, KcGraphInfo, KcParams, KcU128, check

__all__ = ["Context", "Graph", "KCError", "SingleGPU_Kclique", "SingleGPU_Kclique_Local", "parse_spec", "MODES", "UNITS", "ENCODINGS",
           "ORIENTATIONS", "EdgeList", "read_edgelist", "gen_er", "gen_rmat", "gen_chung_lu", "gen_sbm", "gen_batch",
           "batch_count", "footprint_bytes", "lib"]

MODES = {"orient": 0, "orientation": 0, "o": 0, "pivot": 1, "pivoting": 1, "p": 1, "auto": 2}
UNITS = {"node": 0, "edge": 1}
ENCODINGS = {"bitmap": 0, "binary": 0, "b": 0, "list": 1, "n": 1}
ORIENTATIONS = {"degree": 0, "degen": 1, "degeneracy": 1}
FILE_FORMATS = {"auto": 0, "text": 1, "tsv": 1, "mtx": 2, "bel": 3}


def lib():
    return _lib.load()


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _as_u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.uint32)


class Context:
    """One device and one CUDA stream (kc_ctx)."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        check(L.kc_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream_ptr(self) -> int:
        """The cudaStream_t every call of this context runs on (as an int)."""
        s = C.c_void_p()
        check(lib().kc_ctx_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def set_time_limit(self, ns: int) -> None:
        """Device time limit of every counting pass of this context (0 = none);
        a pass past it raises KCError KC_ERR_DEVICE_TIMEOUT."""
        check(lib().kc_ctx_set_time_limit(self._h, int(ns)))

    def set_batch_chunk_edges(self, edges: int) -> None:
        """Host-input batches with more edges than this are counted as a
        pipeline of chunks of whole graphs, the next chunk's copy overlapping
        the current chunk's work (0 = the default, 2**64 - 1 = never)."""
        check(lib().kc_ctx_set_batch_chunk_edges(self._h, int(edges)))

    def close(self):
        if self._h:
            lib().kc_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CountResult:
    count: int
    stats: dict | None = None


class Graph:
    """A device-resident graph (kc_graph)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle

    @classmethod
    def from_edges(cls, ctx: Context, src, dst, n_nodes: int = 0) -> "Graph":
        s, d = _as_u32(src), _as_u32(dst)
        if s.shape != d.shape:
            raise ValueError("src and dst must have the same length")
        h = C.c_void_p()
        check(lib().kc_graph_from_edges(ctx.handle, _u32p(s), _u32p(d), s.size, n_nodes, C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_file(cls, ctx: Context, path, format: str = "auto") -> "Graph":
        """A graph file (text edge list, .mtx or the reference's .bel)."""
        h = C.c_void_p()
        check(lib().kc_graph_from_file(ctx.handle, str(path).encode(), FILE_FORMATS[format], C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_edges_device(cls, ctx: Context, d_src_ptr: int, d_dst_ptr: int, n_edges: int, n_nodes: int = 0):
        h = C.c_void_p()
        check(lib().kc_graph_from_edges_device(ctx.handle, C.c_void_p(d_src_ptr), C.c_void_p(d_dst_ptr), n_edges,
                                               n_nodes, C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_csr(cls, ctx: Context, row_ptr, col_ind) -> "Graph":
        rp, ci = _as_u32(row_ptr), _as_u32(col_ind)
        h = C.c_void_p()
        check(lib().kc_graph_from_csr(ctx.handle, _u32p(rp), _u32p(ci), rp.size - 1, C.byref(h)))
        return cls(ctx, h)

    def close(self):
        if self._h:
            lib().kc_graph_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        i = KcGraphInfo()
        check(lib().kc_graph_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in KcGraphInfo._fields_}

    @property
    def n(self) -> int:
        return self.info()["n"]

    @property
    def m(self) -> int:
        return self.info()["m"]

    def csr(self):
        inf = self.info()
        rp = np.zeros(inf["n"] + 1, np.uint32)
        ci = np.zeros(max(1, 2 * inf["m"]), np.uint32)
        check(lib().kc_graph_get_csr(self._h, _u32p(rp), _u32p(ci)))
        return rp, ci[: 2 * inf["m"]]

    def orient(self, orientation="degree") -> "Graph":
        o = ORIENTATIONS[orientation] if isinstance(orientation, str) else int(orientation)
        check(lib().kc_orient(self._h, o))
        return self

    def dag(self):
        inf = self.info()
        rp = np.zeros(inf["n"] + 1, np.uint32)
        ci = np.zeros(max(1, inf["m"]), np.uint32)
        check(lib().kc_graph_get_dag(self._h, _u32p(rp), _u32p(ci)))
        return rp, ci[: inf["m"]]

    def peel(self):
        n = self.info()["n"]
        prio = np.zeros(max(1, n), np.uint32)
        lev = np.zeros(max(1, n), np.uint32)
        check(lib().kc_graph_get_peel(self._h, _u32p(prio), _u32p(lev)))
        return prio[:n], lev[:n]

    def count(self, k: int, mode="orient", unit="node", part: int = 8, encoding="bitmap",
              stats: bool = False, shard: tuple[int, int] | None = None):
        """Exact number of k-cliques (a Python int; 128-bit on the device).
        shard=(i, S): only unit shard i of S (kc_count_shard); the S shards'
        counts add up to the whole count."""
        p = KcParams()
        p.k = k
        p.mode = MODES[mode] if isinstance(mode, str) else int(mode)
        p.unit = UNITS[unit] if isinstance(unit, str) else int(unit)
        p.part = part
        p.encoding = ENCODINGS[encoding] if isinstance(encoding, str) else int(encoding)
        p.flags = 1 if stats else 0
        out = KcU128()
        st = KcCountStats()
        if shard is None:
            check(lib().kc_count(self._h, C.byref(p), C.byref(out), C.byref(st)))
        else:
            check(lib().kc_count_shard(self._h, C.byref(p), int(shard[0]), int(shard[1]), C.byref(out),
                                       C.byref(st)))
        if stats:
            vals = {f: getattr(st, f) for f, _ in KcCountStats._fields_ if f != "reserved"}
            vals["ms_launch"] = list(vals["ms_launch"])
            vals["cycles"] = list(vals["cycles"])
            return CountResult(out.value(), vals)
        return out.value()

    def count_multi(self, ks, unit="node") -> list:
        """Exact counts for several k in one pivoting walk (kc_count_multi):
        a list in the order of ks."""
        kk = _as_u32(list(ks))
        p = KcParams()
        p.k = int(kk.max()) if kk.size else 0
        p.mode = MODES["pivot"]
        p.unit = UNITS[unit] if isinstance(unit, str) else int(unit)
        p.encoding = ENCODINGS["bitmap"]
        out = (KcU128 * max(1, kk.size))()
        check(lib().kc_count_multi(self._h, C.byref(p), _u32p(kk), kk.size, out))
        return [out[i].value() for i in range(kk.size)]

    def count_local(self, k: int, unit="node", part: int = 8, mode="orient"):
        """Local counts (the reference's -m lkc): a list whose entry v is the
        number of k-cliques containing vertex v; binary encoding."""
        n = self.info()["n"]
        p = KcParams()
        p.k = k
        p.mode = MODES[mode] if isinstance(mode, str) else int(mode)
        p.unit = UNITS[unit] if isinstance(unit, str) else int(unit)
        p.part = part
        p.encoding = ENCODINGS["bitmap"]
        out = (KcU128 * max(1, n))()
        tot = KcU128()
        check(lib().kc_count_local(self._h, C.byref(p), out, C.byref(tot)))
        return [out[v].value() for v in range(n)]

    def kcore(self):
        n = self.info()["n"]
        core = np.zeros(max(1, n), np.uint32)
        mx = C.c_uint32()
        check(lib().kc_kcore(self._h, _u32p(core), C.byref(mx)))
        return core[:n], int(mx.value)

    def truss_support(self) -> np.ndarray:
        m = self.info()["m"]
        sup = np.zeros(max(1, m), np.uint32)
        check(lib().kc_truss_support(self._h, _u32p(sup)))
        return sup[:m]


def parse_spec(spec: str) -> dict:
    """The reference's -q grammar: [o|p]<part>[b|n|h] (include/Config.h:235-271)."""
    p = KcParams()
    check(lib().kc_parse_spec(spec.encode() if spec is not None else None, C.byref(p)))
    return {"mode": int(p.mode), "part": int(p.part), "encoding": int(p.encoding)}


class SingleGPU_Kclique:
    """Mirror of graph::SingleGPU_Kclique<uint> (kclique/kclique.cuh:1302-2643).

    The reference's methods print the count per degree window and return the
    window level from count(); here each method returns the exact k-clique count
    and count() returns the last one.
    """

    def __init__(self, dev: int, g: Graph):
        self.dev = dev
        self.g = g
        self._last = None

    def _run(self, k, unit, mode, enc, part):
        self._last = self.g.count(k, mode=mode, unit=unit, part=part, encoding=enc)
        return self._last

    def findKclqueIncremental_node_async(self, k, part=8):
        return self._run(k, "node", "orient", "list", part)

    def findKclqueIncremental_node_binary_async(self, k, part=8):
        return self._run(k, "node", "orient", "bitmap", part)

    def findKclqueIncremental_node_pivot_async(self, k, part=8):
        return self._run(k, "node", "pivot", "bitmap", part)

    def findKclqueIncremental_node_nobin_pivot_async(self, k, part=8):
        return self._run(k, "node", "pivot", "list", part)

    def findKclqueIncremental_edge_async(self, k, part=8):
        return self._run(k, "edge", "orient", "list", part)

    def findKclqueIncremental_edge_binary_async(self, k, part=8):
        return self._run(k, "edge", "orient", "bitmap", part)

    def findKclqueIncremental_edge_pivot_async(self, k, part=8):
        return self._run(k, "edge", "pivot", "bitmap", part)

    def findKclqueIncremental_edge_nobin_pivot_async(self, k, part=8):
        return self._run(k, "edge", "pivot", "list", part)

    def sync(self):
        return None

    def count(self):
        return self._last


class SingleGPU_Kclique_Local:
    """Mirror of graph::SingleGPU_Kclique_Local<uint> (kclique/kclique_local.cuh:27-639):
    the binary (orientation and pivot) variants; each method returns the
    per-vertex counts (the reference keeps them in its cpn array and prints
    the first 50)."""

    def __init__(self, dev: int, g: Graph):
        self.dev = dev
        self.g = g
        self.cpn = None

    def findKclqueIncremental_node_binary_async_local(self, k, part=8):
        self.cpn = self.g.count_local(k, unit="node", part=part)
        return self.cpn

    def findKclqueIncremental_edge_binary_async_local(self, k, part=8):
        self.cpn = self.g.count_local(k, unit="edge", part=part)
        return self.cpn

    def findKclqueIncremental_node_pivot_async_local(self, k, part=8):
        self.cpn = self.g.count_local(k, unit="node", part=part, mode="pivot")
        return self.cpn

    def findKclqueIncremental_edge_pivot_async_local(self, k, part=8):
        self.cpn = self.g.count_local(k, unit="edge", part=part, mode="pivot")
        return self.cpn


# ---- synthetic inputs ---------------------------------------------------------

class EdgeList:
    """A host edge list owned by the library that made it (optionally page-locked)."""

    def __init__(self, handle, library=None):
        self._h = handle
        self._L = library if library is not None else lib()

    def arrays(self, copy: bool = True):
        s = C.POINTER(C.c_uint32)()
        d = C.POINTER(C.c_uint32)()
        ne = C.c_uint64()
        nn = C.c_uint32()
        check(self._L.kc_edgelist_data(self._h, C.byref(s), C.byref(d), C.byref(ne), C.byref(nn)))
        n = int(ne.value)
        if n == 0:
            return np.zeros(0, np.uint32), np.zeros(0, np.uint32), int(nn.value)
        a = np.ctypeslib.as_array(s, shape=(n,))
        b = np.ctypeslib.as_array(d, shape=(n,))
        if copy:
            a, b = a.copy(), b.copy()
        return a, b, int(nn.value)

    def pointers(self):
        s = C.POINTER(C.c_uint32)()
        d = C.POINTER(C.c_uint32)()
        ne = C.c_uint64()
        nn = C.c_uint32()
        check(self._L.kc_edgelist_data(self._h, C.byref(s), C.byref(d), C.byref(ne), C.byref(nn)))
        return s, d, int(ne.value), int(nn.value)

    def plant_cliques(self, count: int, smin: int, smax: int, seed: int):
        check(self._L.kc_gen_plant_cliques(self._h, count, smin, smax, seed))
        return self

    def batch_meta(self):
        off = C.POINTER(C.c_uint64)()
        nn = C.POINTER(C.c_uint32)()
        kk = C.POINTER(C.c_uint32)()
        fam = C.POINTER(C.c_uint32)()
        ng = C.c_uint32()
        check(self._L.kc_batchgen_meta(self._h, C.byref(off), C.byref(nn), C.byref(kk), C.byref(fam), C.byref(ng)))
        g = int(ng.value)
        return (np.ctypeslib.as_array(off, shape=(g + 1,)).copy(), np.ctypeslib.as_array(nn, shape=(g,)).copy(),
                np.ctypeslib.as_array(kk, shape=(g,)).copy(), np.ctypeslib.as_array(fam, shape=(g,)).copy())

    def close(self):
        if self._h:
            self._L.kc_edgelist_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _gen(fn, *args, library=None) -> EdgeList:
    h = C.c_void_p()
    st = fn(*args, C.byref(h))
    if st != 0:
        L = library if library is not None else lib()
        raise KCError(st, L.kc_last_error().decode(errors="replace"))
    return EdgeList(h, library)


def gen_batch_host(n_graphs: int, base_seed: int, n_min=50, n_max=5000, k_min=4, k_max=12) -> EdgeList:
    """gen_batch through the generator-only library (libkcgen.so): the same
    seeded batch in pageable host memory, for a process that must not load
    the engine."""
    G = _lib.load_gen()
    return _gen(G.kc_gen_batch, n_graphs, base_seed, n_min, n_max, k_min, k_max, 0, library=G)


def read_edgelist(path, format: str = "auto", pinned: bool = False) -> EdgeList:
    """Parses a graph file on host threads (kc_edgelist_from_file)."""
    return _gen(lib().kc_edgelist_from_file, str(path).encode(), FILE_FORMATS[format], int(pinned))


def gen_er(n: int, p: float, seed: int, pinned: bool = False) -> EdgeList:
    return _gen(lib().kc_gen_er, n, p, seed, int(pinned))


def gen_rmat(scale: int, edge_factor: float, a=0.57, b=0.19, c=0.19, seed: int = 1, pinned: bool = False) -> EdgeList:
    return _gen(lib().kc_gen_rmat, scale, edge_factor, a, b, c, seed, int(pinned))


def gen_chung_lu(n: int, exponent: float, mean_degree: float, max_degree: float, seed: int,
                 pinned: bool = False) -> EdgeList:
    return _gen(lib().kc_gen_chung_lu, n, exponent, mean_degree, max_degree, seed, int(pinned))


def gen_sbm(n: int, blocks: int, p_in: float, p_out: float, seed: int, pinned: bool = False) -> EdgeList:
    return _gen(lib().kc_gen_sbm, n, blocks, p_in, p_out, seed, int(pinned))


def gen_batch(n_graphs: int, base_seed: int, n_min=50, n_max=5000, k_min=4, k_max=12, pinned=False) -> EdgeList:
    return _gen(lib().kc_gen_batch, n_graphs, base_seed, n_min, n_max, k_min, k_max, int(pinned))


def footprint_bytes(n_nodes: int, n_edges: int, max_out: int) -> int:
    return int(lib().kc_footprint_bytes(n_nodes, n_edges, max_out))


def _u128_list(arr, n: int) -> list:
    """Python ints from a ctypes array of kc_u128 (numpy for the common case
    where no count needs the high word)."""
    if n == 0:
        return []
    w = np.frombuffer(arr, dtype=np.uint64, count=2 * n).reshape(n, 2)
    if not w[:, 1].any():
        return w[:, 0].tolist()
    return [(int(h) << 64) | int(lo) for lo, h in w.tolist()]


def _params(d: dict) -> KcParams:
    p = KcParams()
    for key, table in (("mode", MODES), ("unit", UNITS), ("encoding", ENCODINGS)):
        v = d.get(key, 0)
        setattr(p, key, table[v] if isinstance(v, str) else int(v))
    p.part = int(d.get("part", 0))
    return p


def batch_count(ctx: Context, src, dst, edge_off, n_nodes, ks, orientation="degree", autotune=True,
                fixed: dict | None = None, use_graph=True, return_choice=False, return_stats=False,
                device_ptrs: tuple | None = None, graph_params: list | None = None):
    """Counts a packed batch: graph i owns edges [edge_off[i], edge_off[i+1]).

    With device_ptrs=(d_src, d_dst) the edges are read from device memory of
    the context's GPU (src/dst are then ignored). graph_params: a method per
    graph (dicts of mode / unit / part / encoding) instead of the autotuner."""
    if device_ptrs is None:
        s, d = _as_u32(src), _as_u32(dst)
    off = np.ascontiguousarray(edge_off, dtype=np.uint64)
    nn = _as_u32(n_nodes)
    kk = _as_u32(ks)
    g = nn.size
    opts = KcBatchOpts()
    opts.orientation = ORIENTATIONS[orientation] if isinstance(orientation, str) else int(orientation)
    opts.autotune = 1 if autotune else 0
    opts.use_graph = 1 if use_graph else 0
    opts.flags = 1 if return_stats else 0
    if fixed:
        opts.fixed.mode = MODES.get(fixed.get("mode", "orient"), 0) if isinstance(fixed.get("mode"), str) else int(fixed.get("mode", 0))
        opts.fixed.unit = UNITS.get(fixed.get("unit", "node"), 0) if isinstance(fixed.get("unit"), str) else int(fixed.get("unit", 0))
        opts.fixed.part = int(fixed.get("part", 8))
        opts.fixed.encoding = ENCODINGS.get(fixed.get("encoding", "bitmap"), 0) if isinstance(fixed.get("encoding"), str) else int(fixed.get("encoding", 0))
    if graph_params is not None:
        gp = (KcParams * max(1, g))(*[_params(x) for x in graph_params])
        opts.graph_params = C.cast(gp, C.c_void_p)
    counts = (KcU128 * g)()
    choice = (KcParams * g)()
    st = KcBatchStats()
    offp = off.ctypes.data_as(C.POINTER(C.c_uint64))
    if device_ptrs is None:
        check(lib().kc_batch_count_packed(ctx.handle, _u32p(s), _u32p(d), offp, _u32p(nn), _u32p(kk), g,
                                          C.byref(opts), counts, choice, C.byref(st)))
    else:
        check(lib().kc_batch_count_packed_device(ctx.handle, C.c_void_p(device_ptrs[0]), C.c_void_p(device_ptrs[1]),
                                                 offp, _u32p(nn), _u32p(kk), g, C.byref(opts), counts, choice,
                                                 C.byref(st)))
    res = _u128_list(counts, g)
    out = [res]
    if return_choice:
        out.append([{"mode": int(c.mode), "unit": int(c.unit), "part": int(c.part), "encoding": int(c.encoding)}
                    for c in choice])
    if return_stats:
        vals = {f: getattr(st, f) for f, _ in KcBatchStats._fields_}
        vals["cycles"] = list(vals["cycles"])
        vals["host_ms"] = list(vals["host_ms"])
        out.append(vals)
    return out[0] if len(out) == 1 else tuple(out)


# ---- serving -------------------------------------------------------------------

class Server:
    """Continuous-batching request server (kc_server): requests of different
    graphs and k run on several device streams as slots and HBM free up."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 0, streams: int = 4, orientation="degen",
                 autotune: bool = True, fixed: dict | None = None):
        o = _lib.KcServerOpts()
        o.hbm_budget_bytes = int(hbm_budget_bytes)
        o.streams = int(streams)
        o.max_inflight = int(streams)
        o.orientation = ORIENTATIONS[orientation] if isinstance(orientation, str) else int(orientation)
        o.autotune = 1 if autotune else 0
        if fixed:
            o.fixed.mode = MODES[fixed.get("mode", "pivot")]
            o.fixed.unit = UNITS[fixed.get("unit", "node")]
            o.fixed.part = int(fixed.get("part", 8))
            o.fixed.encoding = ENCODINGS[fixed.get("encoding", "bitmap")]
        h = C.c_void_p()
        check(lib().kc_server_create(ctx.handle, C.byref(o), C.byref(h)))
        self._h = h
        self.ctx = ctx

    def put_graph(self, src, dst, n_nodes: int = 0) -> int:
        s, d = _as_u32(src), _as_u32(dst)
        gid = C.c_uint64()
        check(lib().kc_server_put_graph(self._h, _u32p(s), _u32p(d), s.size, n_nodes, C.byref(gid)))
        return int(gid.value)

    def drop_graph(self, graph_id: int) -> None:
        check(lib().kc_server_drop_graph(self._h, graph_id))

    def submit(self, graph_id: int, k: int) -> int:
        t = C.c_uint64()
        check(lib().kc_server_submit(self._h, graph_id, k, C.byref(t)))
        return int(t.value)

    def submit_edges(self, src, dst, n_nodes: int, k: int) -> int:
        s, d = _as_u32(src), _as_u32(dst)
        t = C.c_uint64()
        check(lib().kc_server_submit_edges(self._h, _u32p(s), _u32p(d), s.size, n_nodes, k, C.byref(t)))
        return int(t.value)

    def cancel(self, ticket: int) -> None:
        check(lib().kc_server_cancel(self._h, ticket))

    def wait(self, ticket: int, wait_ms: int = -1) -> dict:
        r = _lib.KcRequestResult()
        check(lib().kc_server_wait(self._h, ticket, wait_ms, C.byref(r)))
        return {"count": r.count.value(), "status": int(r.status), "k": int(r.k), "submit_ms": r.submit_ms,
                "start_ms": r.start_ms, "done_ms": r.done_ms, "graph_id": int(r.graph_id),
                "params": {"mode": int(r.params.mode), "unit": int(r.params.unit), "part": int(r.params.part),
                           "encoding": int(r.params.encoding)}}

    def close(self):
        if self._h:
            lib().kc_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
