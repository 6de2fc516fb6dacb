#!/usr/bin/env bash
# Builds the reference's own k-clique program (KCGPU, src/main.cu) for sm_100a
# into oracle/_ref/kcgpu_ref. TEST INFRASTRUCTURE: the binary is run only by
# tests/golden/make_ref_golden.py to record golden counts; nothing in the
# engine, the tests' GPU path or bench.py runs it.
#
# The reference's sources are compiled where they lie, unmodified, through a
# tree of per-file symbolic links (oracle/_ref/tree). Two things differ from
# its own Makefile (sm_70/75, CUDA 10-era):
#  * its vendored 2018 CUB (cub/) uses texture references, which CUDA 12
#    removed, so tree/cub/cub.cuh is a two-line header that includes the
#    toolkit's CUB instead; the reference reaches CUB only through
#    include/utils.cuh:27 ("../cub/cub.cuh"), which resolves to that header
#    inside the tree;
#  * oracle/ref_shim.cu is linked in with ld --wrap (its header says why).
# Usage: bash oracle/build_ref.sh [reference root]   (default: $KC_REFERENCE
# or /root/reference). Exits 0 without building when the sources are absent.
set -euo pipefail
REF="${1:-${KC_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/main.cu" ]; then
  echo "build_ref: reference sources not found at $REF; nothing built"
  exit 0
fi
NVCC="${NVCC:-nvcc}"
command -v "$NVCC" >/dev/null || NVCC=/usr/local/cuda/bin/nvcc
ARCH=(-gencode arch=compute_100a,code=sm_100a)
BIN="$OUT/kcgpu_ref"

# up to date: the binary is newer than every reference source and the shim
if [ -x "$BIN" ] && [ -z "$(find "$REF/src" "$REF/include" "$REF/kclique" "$REF/kcore" "$REF/truss" \
      "$HERE/ref_shim.cu" "$HERE/build_ref.sh" -newer "$BIN" -print -quit 2>/dev/null)" ]; then
  echo "build_ref: $BIN is up to date"
  exit 0
fi

rm -rf "$OUT/tree"
mkdir -p "$OUT/tree/cub"
for d in src include kclique kcore truss; do
  mkdir -p "$OUT/tree/$d"
  for f in "$REF/$d"/*; do ln -s "$f" "$OUT/tree/$d/"; done
done
printf '#pragma once\n#include <cub/cub.cuh>\n' > "$OUT/tree/cub/cub.cuh"

# the reference's own flags (-w -lineinfo -O3 -DCUDA -DNOT_IMPL), C++17 for
# the toolkit's CUB, sm_100a, OpenMP as its host code uses it
"$NVCC" -w -lineinfo -std=c++17 -O3 -DCUDA -DNOT_IMPL "${ARCH[@]}" -Xcompiler -fopenmp \
  -c "$OUT/tree/src/main.cu" -o "$OUT/main.o"
"$NVCC" -O2 -std=c++17 "${ARCH[@]}" -c "$HERE/ref_shim.cu" -o "$OUT/ref_shim.o"
"$NVCC" "${ARCH[@]}" -o "$BIN.tmp" "$OUT/main.o" "$OUT/ref_shim.o" \
  -Xlinker --wrap=fopen -Xlinker --wrap=cudaGetDeviceProperties_v2 -Xcompiler -fopenmp
mv "$BIN.tmp" "$BIN"
# only the binary stays: the link tree points into the reference checkout,
# which the GPU machines do not have
rm -rf "$OUT/tree" "$OUT/main.o" "$OUT/ref_shim.o"
echo "build_ref: built $BIN"
