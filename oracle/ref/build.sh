#!/bin/sh
# Builds, from the reference's own sources where they lie in the reference
# tree (REF_ROOT; by default the directory `reference` beside the checkout of
# this repository):
#   oracle/_ref/libref_tritri.so -- the gProximity triangle-pair predicate;
#   oracle/_ref/ref_emu_driver   -- the reference's collision pipeline as host
#                                   C++ (Makefile.refemu).
# Output goes to oracle/_ref/ only.  Skips quietly when the
# reference tree is absent (the GPU box has only the prebuilt files).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF_ROOT=${REF_ROOT:-$(cd "$HERE/../../.." && pwd)/reference}
OUT="$HERE/../_ref"
GP="$REF_ROOT/Source/Externals/inc/gProximity"
if [ ! -f "$GP/cuda_intersect_tritri.h" ]; then
  echo "reference tree not found at $REF_ROOT; oracle/_ref not rebuilt"
  exit 0
fi
mkdir -p "$OUT"
CUDA_INC=${CUDA_HOME:-/usr/local/cuda}/include
g++ -O2 -std=c++17 -fPIC -shared -ffp-contract=off -w \
    -I"$GP" -I"$CUDA_INC" "$HERE/gproximity_tritri.cpp" -o "$OUT/libref_tritri.so"
echo "built $OUT/libref_tritri.so"
make -s -j8 -f "$HERE/Makefile.refemu" REF_ROOT="$REF_ROOT"
echo "built $OUT/ref_emu_driver"
