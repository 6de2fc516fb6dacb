"""ctypes binding of libkc.so (the C ABI declared in include/kc.h).

The library is loaded from the package directory only; if it is missing the
import fails loudly (there is no CPU fallback for any engine call).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libkc.so"

u32, u64, i32, i64 = C.c_uint32, C.c_uint64, C.c_int, C.c_int64
P = C.POINTER


class KcU128(C.Structure):
    _fields_ = [("lo", u64), ("hi", u64)]

    def value(self) -> int:
        return (int(self.hi) << 64) | int(self.lo)


class KcParams(C.Structure):
    _fields_ = [("k", u32), ("mode", u32), ("unit", u32), ("part", u32), ("encoding", u32), ("flags", u32)]


class KcCountStats(C.Structure):
    _fields_ = [("units", u64), ("tree_nodes", u64), ("word_ops", u64), ("gather_bytes", u64),
                ("ms_total", C.c_double), ("ms_traversal", C.c_double), ("max_unit_size", u32),
                ("kernels", u32), ("ms_launch", C.c_double * 5), ("heavy_units", u64), ("deep_retry", u32),
                ("reserved", u32), ("cycles", u64 * 3)]


class KcGraphInfo(C.Structure):
    _fields_ = [("n", u32), ("m", u64), ("max_degree", u32), ("oriented", u32), ("max_out_degree", u32),
                ("max_core", u32), ("device_bytes", u64)]


class KcBatchGraph(C.Structure):
    _fields_ = [("src", P(u32)), ("dst", P(u32)), ("n_edges", u64), ("n_nodes", u32), ("k", u32)]


class KcBatchOpts(C.Structure):
    _fields_ = [("orientation", u32), ("autotune", u32), ("fixed", KcParams), ("use_graph", u32),
                ("flags", u32), ("graph_params", C.c_void_p)]


class KcBatchStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_h2d", C.c_double), ("ms_build", C.c_double),
                ("ms_count", C.c_double), ("units", u64), ("kernels", u32), ("n_graphs", u32),
                ("tree_nodes", u64), ("word_ops", u64), ("gather_bytes", u64), ("heavy_units", u64),
                ("cycles", u64 * 3), ("ms_csr", C.c_double), ("ms_orient", C.c_double),
                ("host_ms", C.c_double * 5), ("n_vertices", u64), ("n_edges", u64)]


class KcServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", u64), ("max_inflight", u32), ("streams", u32), ("orientation", u32),
                ("autotune", u32), ("fixed", KcParams)]


class KcRequestResult(C.Structure):
    _fields_ = [("count", KcU128), ("status", i32), ("k", u32), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("done_ms", C.c_double), ("graph_id", u64), ("params", KcParams)]


# name -> (restype, argtypes)
SIGNATURES = {
    "kc_ctx_create": (i32, [i32, P(C.c_void_p)]),
    "kc_ctx_destroy": (i32, [C.c_void_p]),
    "kc_last_error": (C.c_char_p, []),
    "kc_status_string": (C.c_char_p, [i32]),
    "kc_ctx_set_time_limit": (i32, [C.c_void_p, u64]),
    "kc_ctx_set_batch_chunk_edges": (i32, [C.c_void_p, u64]),
    "kc_ctx_release_cached_memory": (i32, [C.c_void_p]),
    "kc_ctx_get_stream": (i32, [C.c_void_p, P(C.c_void_p)]),
    "kc_kernel_launches": (u64, []),
    "kc_test_fail_alloc_after": (None, [i64]),
    "kc_test_live_allocations": (u64, []),
    "kc_graph_from_edges": (i32, [C.c_void_p, P(u32), P(u32), u64, u32, P(C.c_void_p)]),
    "kc_graph_from_edges_device": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, u32, P(C.c_void_p)]),
    "kc_graph_from_csr": (i32, [C.c_void_p, P(u32), P(u32), u32, P(C.c_void_p)]),
    "kc_graph_destroy": (i32, [C.c_void_p]),
    "kc_graph_get_info": (i32, [C.c_void_p, P(KcGraphInfo)]),
    "kc_graph_get_csr": (i32, [C.c_void_p, P(u32), P(u32)]),
    "kc_orient": (i32, [C.c_void_p, u32]),
    "kc_graph_get_dag": (i32, [C.c_void_p, P(u32), P(u32)]),
    "kc_graph_get_peel": (i32, [C.c_void_p, P(u32), P(u32)]),
    "kc_count": (i32, [C.c_void_p, P(KcParams), P(KcU128), P(KcCountStats)]),
    "kc_count_shard": (i32, [C.c_void_p, P(KcParams), u32, u32, P(KcU128), P(KcCountStats)]),
    "kc_count_multi": (i32, [C.c_void_p, P(KcParams), P(u32), u32, P(KcU128)]),
    "kc_count_local": (i32, [C.c_void_p, P(KcParams), P(KcU128), P(KcU128)]),
    "kc_parse_spec": (i32, [C.c_char_p, P(KcParams)]),
    "kc_kcore": (i32, [C.c_void_p, P(u32), P(u32)]),
    "kc_truss_support": (i32, [C.c_void_p, P(u32)]),
    "kc_truss_support_noalloc": (i32, [C.c_void_p, C.c_void_p, u32, C.c_void_p, C.c_void_p]),
    "kc_batch_count": (i32, [C.c_void_p, P(KcBatchGraph), u32, P(KcBatchOpts), P(KcU128), P(KcParams),
                             P(KcBatchStats)]),
    "kc_batch_count_packed": (i32, [C.c_void_p, P(u32), P(u32), P(u64), P(u32), P(u32), u32, P(KcBatchOpts),
                                    P(KcU128), P(KcParams), P(KcBatchStats)]),
    "kc_batch_count_packed_device": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, P(u64), P(u32), P(u32), u32,
                                           P(KcBatchOpts), P(KcU128), P(KcParams), P(KcBatchStats)]),
    "kc_server_create": (i32, [C.c_void_p, P(KcServerOpts), P(C.c_void_p)]),
    "kc_server_destroy": (i32, [C.c_void_p]),
    "kc_server_put_graph": (i32, [C.c_void_p, P(u32), P(u32), u64, u32, P(u64)]),
    "kc_server_drop_graph": (i32, [C.c_void_p, u64]),
    "kc_server_submit": (i32, [C.c_void_p, u64, u32, P(u64)]),
    "kc_server_submit_edges": (i32, [C.c_void_p, P(u32), P(u32), u64, u32, u32, P(u64)]),
    "kc_server_cancel": (i32, [C.c_void_p, u64]),
    "kc_server_wait": (i32, [C.c_void_p, u64, i64, P(KcRequestResult)]),
    "kc_footprint_bytes": (u64, [u32, u64, u32]),
    "kc_edgelist_data": (i32, [C.c_void_p, P(P(u32)), P(P(u32)), P(u64), P(u32)]),
    "kc_edgelist_destroy": (i32, [C.c_void_p]),
    "kc_edgelist_from_file": (i32, [C.c_char_p, u32, i32, P(C.c_void_p)]),
    "kc_graph_from_file": (i32, [C.c_void_p, C.c_char_p, u32, P(C.c_void_p)]),
    "kc_gen_er": (i32, [u32, C.c_double, u64, i32, P(C.c_void_p)]),
    "kc_gen_rmat": (i32, [u32, C.c_double, C.c_double, C.c_double, C.c_double, u64, i32, P(C.c_void_p)]),
    "kc_gen_chung_lu": (i32, [u32, C.c_double, C.c_double, C.c_double, u64, i32, P(C.c_void_p)]),
    "kc_gen_sbm": (i32, [u32, u32, C.c_double, C.c_double, u64, i32, P(C.c_void_p)]),
    "kc_gen_plant_cliques": (i32, [C.c_void_p, u32, u32, u32, u64]),
    "kc_gen_batch": (i32, [u32, u64, u32, u32, u32, u32, i32, P(C.c_void_p)]),
    "kc_batchgen_meta": (i32, [C.c_void_p, P(P(u64)), P(P(u32)), P(P(u32)), P(P(u32)), P(u32)]),
}

STATUS = {0: "KC_OK", 1: "KC_ERR_INVALID_ARG", 2: "KC_ERR_OOM", 3: "KC_ERR_ADMISSION", 4: "KC_ERR_DEVICE_TIMEOUT",
          5: "KC_ERR_CUDA", 6: "KC_ERR_INTERNAL", 7: "KC_ERR_NOT_ORIENTED", 8: "KC_ERR_CANCELLED", 9: "KC_ERR_BUSY"}


class KCError(RuntimeError):
    """A failing engine call: .status is the kc_status code, .name its name."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


_lib = None


def load(path: Path | None = None) -> C.CDLL:
    """Loads libkc.so (once) and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    # KC_LIBRARY names another build of the engine in this package (tests load
    # the bounds-checked libkc_checked.so that way)
    alt = os.environ.get("KC_LIBRARY")
    p = Path(path) if path else (_LIB_PATH.parent / alt if alt else _LIB_PATH)
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m kcgpu_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


_gen_lib = None
_GEN_PATH = Path(__file__).resolve().parent / "libkcgen.so"
_GEN_SIGNATURES = ("kc_last_error", "kc_edgelist_data", "kc_edgelist_destroy", "kc_gen_er", "kc_gen_rmat",
                   "kc_gen_chung_lu", "kc_gen_sbm", "kc_gen_plant_cliques", "kc_gen_batch", "kc_batchgen_meta")


def load_gen() -> C.CDLL:
    """Loads libkcgen.so (the seeded generators without the engine) once."""
    global _gen_lib
    if _gen_lib is None:
        if not _GEN_PATH.exists():
            raise ImportError(f"{_GEN_PATH} is missing: build it with `python -m kcgpu_b200.build`")
        g = C.CDLL(str(_GEN_PATH))
        for name in _GEN_SIGNATURES:
            f = getattr(g, name)
            f.restype, f.argtypes = SIGNATURES[name]
        _gen_lib = g
    return _gen_lib


def check(status: int) -> None:
    if status != 0:
        msg = _lib.kc_last_error().decode(errors="replace") if _lib is not None else ""
        raise KCError(status, msg)
