#!/usr/bin/env bash
# Builds kadircs/hmglib's own CUDA sources (read in place from the reference
# checkout) for sm_100a into oracle/_ref/, with the MAGMA stand-in of this folder,
# plus the ref_dump driver.  TEST INFRASTRUCTURE ONLY: the result is the oracle the
# parity fixtures are generated with; the product never links it.
#
# usage: oracle/refbuild/build_ref.sh REFERENCE_SRC_DIR
#    or: HMG_REFERENCE_SRC=REFERENCE_SRC_DIR oracle/refbuild/build_ref.sh
# (REFERENCE_SRC_DIR is the reference checkout's src/ folder)
#
# Needed deviations from the reference's own Makefile (src/Makefile:19-71):
#   * MAGMA is neither installed nor vendored -> magma_v2.h / magma_lapack.h /
#     magma_shim.cu here;
#   * tree.cu relies on thrust/remove.h arriving through another header, which the
#     CUDA 12.9 Thrust no longer does -> -include thrust/remove.h;
#   * src/ must not be on the include path (its vendored CUB 1.x shadows the
#     toolkit's and fails Thrust's version check) -> the headers the dump program needs
#     are linked into oracle/_ref/include instead;
#   * sm_100a instead of sm_61, no -G.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${HMG_REFERENCE_SRC:-}}"
if [ -z "$REF" ] || [ ! -d "$REF" ]; then
  echo "usage: $0 REFERENCE_SRC_DIR (or set HMG_REFERENCE_SRC)" >&2
  exit 2
fi
OUT="$HERE/../_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
mkdir -p "$OUT/obj" "$OUT/include"
for h in hmglib.h morton.h tree.h linear_algebra.h system_assembler.h kernel_system_assembler.h helper.h; do
  ln -sf "$REF/$h" "$OUT/include/$h"
done
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O2 -rdc=true -std=c++17 -w
       -include thrust/remove.h -I "$HERE" -I "$OUT/include" -Xcompiler -fPIC)
objs=()
for s in helper hmglib kernel_system_assembler linear_algebra morton tree; do
  "$NVCC" "${FLAGS[@]}" -c "$REF/$s.cu" -o "$OUT/obj/$s.o"
  objs+=("$OUT/obj/$s.o")
done
"$NVCC" "${FLAGS[@]}" -c "$HERE/magma_shim.cu" -o "$OUT/obj/magma_shim.o"
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_dump.cu" -o "$OUT/obj/ref_dump.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -rdc=true -o "$OUT/ref_dump" \
  "${objs[@]}" "$OUT/obj/magma_shim.o" "$OUT/obj/ref_dump.o" -lcublas -lcurand
rm -rf "$OUT/obj" "$OUT/include"
echo "$OUT/ref_dump"
