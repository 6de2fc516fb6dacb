"""Builds the engine's shared library in-tree: kcgpu_b200/libkc.so.

Every CUDA translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), with line info for profiling.
Objects go to kcgpu_b200/_build/ and are rebuilt when their source or any
header is newer. Run ``python -m kcgpu_b200.build`` or call ``build()``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libkc.so"
GEN_LIB = PKG / "libkcgen.so"
CHECKED_LIB = PKG / "libkc_checked.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3"] + ARCH


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the engine has no CPU fallback and needs the CUDA toolkit to build")


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _compile(nvcc: str, src: Path, verbose: bool, bdir: Path = BUILD, extra: tuple = ()) -> Path:
    obj = bdir / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc] + NVCC_FLAGS + list(extra) + ["-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[1:1] = ["-x", "cu"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None, checked: bool = False) -> Path:
    """Compiles every source under csrc/ and links libkc.so; returns its path.

    checked=True builds libkc_checked.so instead: the same engine compiled
    with -DKC_CHECKED, whose kernels check their data-dependent scratch
    indices, record DEV_ERR_BOUNDS and skip the access (tests load it through
    the KC_LIBRARY environment variable)."""
    nvcc = _nvcc()
    bdir = BUILD / "checked" if checked else BUILD
    lib = CHECKED_LIB if checked else LIB
    extra = ("-DKC_CHECKED",) if checked else ()
    bdir.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(nvcc, s, verbose, bdir, extra), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    LIB_ = lib
    if not LIB_.exists() or LIB_.stat().st_mtime < newest:
        tmp = LIB_.with_suffix(".so.tmp")
        # launches are counted (engine.cu) and device allocations pass the
        # fault-injection hook (alloc_hook.cpp)
        wrapped = ["cudaLaunchKernel", "cudaLaunchCooperativeKernel", "cudaMalloc", "cudaMallocAsync", "cudaFree",
                   "cudaFreeAsync"]
        wrap = [x for f in wrapped for x in ("-Xlinker", f"--wrap={f}")]
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + wrap + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking {LIB_.name} failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB_)
    if checked:
        return LIB_
    # the seeded input generators alone, for processes that must not load the
    # engine (the CPU reference arm of bench.py)
    gen_objs = [BUILD / "gen.cpp.o", BUILD / "errors.cpp.o"]
    if not GEN_LIB.exists() or GEN_LIB.stat().st_mtime < max(o.stat().st_mtime for o in gen_objs):
        tmp = GEN_LIB.with_suffix(".so.tmp")
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in gen_objs] + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking libkcgen.so failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, GEN_LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, checked="--checked" in sys.argv))
