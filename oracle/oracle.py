"""ctypes front end of the CPU oracle (oracle.cpp). TEST INFRASTRUCTURE.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module;
the engine never does. See oracle.cpp for the reference lines each rule
follows.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_lib = None
P = C.POINTER
u32, u64 = C.c_uint32, C.c_uint64


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.or_from_edges.restype = C.c_void_p
        L.or_from_edges.argtypes = [P(u32), P(u32), u64, u32]
        L.or_from_csr.restype = C.c_void_p
        L.or_from_csr.argtypes = [P(u32), P(u32), u32]
        L.or_free.argtypes = [C.c_void_p]
        L.or_n.restype = u32
        L.or_n.argtypes = [C.c_void_p]
        L.or_m.restype = u64
        L.or_m.argtypes = [C.c_void_p]
        L.or_get_csr.argtypes = [C.c_void_p, P(u32), P(u32)]
        L.or_max_degree.restype = u32
        L.or_max_degree.argtypes = [C.c_void_p]
        L.or_orient.restype = u32
        L.or_orient.argtypes = [C.c_void_p, C.c_int]
        L.or_get_dag.argtypes = [C.c_void_p, P(u32), P(u32)]
        L.or_get_peel.argtypes = [C.c_void_p, P(u32), P(u32)]
        L.or_kcore.restype = u32
        L.or_kcore.argtypes = [C.c_void_p, P(u32)]
        L.or_count.restype = C.c_int
        L.or_count.argtypes = [C.c_void_p, u32, C.c_int, C.c_int, C.c_int, P(u64), P(u64)]
        L.or_count_ex.restype = C.c_int
        L.or_count_ex.argtypes = [C.c_void_p, u32, C.c_int, C.c_int, C.c_int, C.c_int, P(u64), P(u64)]
        L.or_truss_support.argtypes = [C.c_void_p, P(u32)]
        L.or_count_local.restype = C.c_int
        L.or_count_local.argtypes = [C.c_void_p, u32, P(u64), P(u64)]
        L.or_binom.argtypes = [u32, u32, P(u64), P(u64)]
        L.or_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(P(u32))


class OracleGraph:
    """Symmetric, deduplicated CSR on the host plus the reference's orientation rules."""

    def __init__(self, src, dst, n_nodes: int = 0):
        L = load()
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        self._h = L.or_from_edges(_p(s), _p(d), s.size, n_nodes)

    def __del__(self):
        if getattr(self, "_h", None):
            load().or_free(self._h)
            self._h = None

    @property
    def n(self) -> int:
        return int(load().or_n(self._h))

    @property
    def m(self) -> int:
        return int(load().or_m(self._h))

    def csr(self):
        rp = np.zeros(self.n + 1, np.uint32)
        ci = np.zeros(max(1, 2 * self.m), np.uint32)
        load().or_get_csr(self._h, _p(rp), _p(ci))
        return rp, ci[: 2 * self.m]

    def max_degree(self) -> int:
        return int(load().or_max_degree(self._h))

    def orient(self, orientation: str = "degree") -> int:
        """Returns the largest out-degree."""
        return int(load().or_orient(self._h, 1 if orientation.startswith("degen") else 0))

    def dag(self):
        rp = np.zeros(self.n + 1, np.uint32)
        ci = np.zeros(max(1, self.m), np.uint32)
        load().or_get_dag(self._h, _p(rp), _p(ci))
        return rp, ci[: self.m]

    def peel(self):
        prio = np.zeros(max(1, self.n), np.uint32)
        lev = np.zeros(max(1, self.n), np.uint32)
        load().or_get_peel(self._h, _p(prio), _p(lev))
        return prio[: self.n], lev[: self.n]

    def kcore(self):
        core = np.zeros(max(1, self.n), np.uint32)
        mx = load().or_kcore(self._h, _p(core))
        return core[: self.n], int(mx)

    def count(self, k: int, mode: str = "orient", unit: str = "node", threads: int = 0,
              closed: bool = False) -> int:
        """closed (pivoting only): end clique-tree nodes with k - held <= 2 by
        their closed form instead of expanding them; same count, faster."""
        lo, hi = u64(), u64()
        rc = load().or_count_ex(self._h, k, 1 if mode.startswith("p") else 0, 1 if unit == "edge" else 0, threads,
                                1 if closed else 0, C.byref(lo), C.byref(hi))
        if rc != 0:
            raise RuntimeError("oracle count failed (graph not oriented or k == 0)")
        return (int(hi.value) << 64) | int(lo.value)

    def count_local(self, k: int) -> list:
        """Per-vertex k-clique counts (every clique credits each of its vertices)."""
        lo = np.zeros(max(1, self.n), np.uint64)
        hi = np.zeros(max(1, self.n), np.uint64)
        rc = load().or_count_local(self._h, k, lo.ctypes.data_as(P(u64)), hi.ctypes.data_as(P(u64)))
        if rc != 0:
            raise RuntimeError("oracle local count failed (graph not oriented or k == 0)")
        return [(int(h) << 64) | int(l) for l, h in zip(lo[: self.n], hi[: self.n])]

    def truss_support(self) -> np.ndarray:
        sup = np.zeros(max(1, self.m), np.uint32)
        load().or_truss_support(self._h, _p(sup))
        return sup[: self.m]


def binom(n: int, r: int) -> int:
    lo, hi = u64(), u64()
    load().or_binom(n, r, C.byref(lo), C.byref(hi))
    return (int(hi.value) << 64) | int(lo.value)


def max_threads() -> int:
    return int(load().or_max_threads())
