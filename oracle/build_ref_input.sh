#!/usr/bin/env bash
# Builds the reference's own input path for the host, as the checker of the
# real-topology builder (lima_topology_*):
#   oracle/_ref/lima_ref_ffmaker  LIMA_ForcefieldMaker/LIMA_ForcefieldMaker.cpp
#                                 compiled unchanged
#   oracle/_ref/lima_ref_boxdump  oracle/ref_input_driver.cpp with the
#                                 reference's CompoundBuilder.cpp, Forcefield.cu,
#                                 BoxBuilder.cu, Bodies.cu, Filehandling.cpp and
#                                 QuantomTypes.cu compiled as host C++ (CUDA
#                                 qualifiers from oracle/ref_shim)
# The reference sources are read from $LIMA_REF_ROOT (default /root/reference)
# and copied to a temporary directory outside the repository; they are not
# modified.  Test infrastructure: the product never runs these programs.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${LIMA_REF_ROOT:-/root/reference}"
SRC="$REF_ROOT/Quantom/Quantom"
FFM="$REF_ROOT/LIMA_ForcefieldMaker/LIMA_ForcefieldMaker"
OUT="$HERE/_ref"
if [ ! -f "$SRC/CompoundBuilder.cpp" ] || [ ! -f "$FFM/LIMA_ForcefieldMaker.cpp" ]; then
    echo "build_ref_input.sh: reference sources not found under $REF_ROOT; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d /tmp/lima_ref_input.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT
for f in CompoundBuilder.cpp CompoundBuilder.h Forcefield.cu Forcefield.cuh BoxBuilder.cu BoxBuilder.cuh Bodies.cu \
         Bodies.cuh Filehandling.cpp Filehandling.h QuantomTypes.cu QuantomTypes.cuh Simulation.cuh Constants.cuh; do
    cp "$SRC/$f" "$TMP/$f"
done
CXX="${CXX:-g++}"
"$CXX" -std=c++17 -O2 -w "$FFM/LIMA_ForcefieldMaker.cpp" -I"$FFM" -o "$OUT/lima_ref_ffmaker.tmp"
mv "$OUT/lima_ref_ffmaker.tmp" "$OUT/lima_ref_ffmaker"
"$CXX" -std=c++17 -O2 -w -I"$TMP" -I"$HERE/ref_shim" \
    -include "$HERE/ref_shim/cuda_runtime.h" -include "$HERE/ref_shim/input_extra.h" \
    -x c++ "$HERE/ref_input_driver.cpp" "$TMP/CompoundBuilder.cpp" "$TMP/Forcefield.cu" "$TMP/BoxBuilder.cu" \
    "$TMP/Bodies.cu" "$TMP/Filehandling.cpp" "$TMP/QuantomTypes.cu" -o "$OUT/lima_ref_boxdump.tmp"
mv "$OUT/lima_ref_boxdump.tmp" "$OUT/lima_ref_boxdump"
echo "built $OUT/lima_ref_ffmaker $OUT/lima_ref_boxdump"
