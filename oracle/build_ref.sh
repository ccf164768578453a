#!/usr/bin/env bash
# Builds oracle/_ref/libref_lima.so: the reference LIMA_MD engine's own
# per-step code (Quantom/Quantom/Engine.cu + headers) compiled for the host CPU
# together with the block emulator in oracle/ref_emu.cpp.  Test
# infrastructure: the product never loads this library.
#
# The reference sources are read from $LIMA_REF_ROOT (default /root/reference)
# and copied to a temporary directory OUTSIDE the repository, where five
# documented changes are made before compiling; only the built .so is written
# under oracle/_ref/:
#   1. Constants.cuh is replaced by oracle/ref_shim/Constants.cuh (runtime box
#      length and cutoff, raised list capacities);
#   2. Bodies.cuh: the second `i += blockDim.x;` in NeighborList::loadData
#      (Bodies.cuh:282) is deleted, so every solvent id is staged;
#   3. Engine.cu: Engine::step (Engine.cu:400-451, CUDA launch syntax) is
#      deleted; ref_emu.cpp defines it with emulated launches;
#   4. Engine.cu: integratePosition (Engine.cu:849) gets one call to
#      lima_ref_force_hook(p_index, force) as its first statement;
#   5. Engine.cu: a __syncthreads() after the shared accumulator reset at the
#      top of computePairbondForces/AnglebondForces/DihedralForces
#      (Engine.cu:746,779,814), and one between thread 0's applyPBC of
#      particle 0 and the other threads' applyHyperpos to it (Engine.cu:993-996).
#      The reference has no barrier at either point; on a GPU, warp 0 executes
#      them in program order (every lane resets before lane 0 adds; lanes read
#      particle 0 after lane 0 wrapped it).  The host emulator runs threads one
#      after another, so without the barriers it would resolve both races
#      differently from the hardware.
# The rasterizer (Quantom/Quantom/Rasterizer.cu + .cuh) is compiled in as well,
# with two changes to the copy:
#   6. the Rasterizer member functions render/getAllAtoms/sortAtoms/
#      processAtoms (Rasterizer.cu:12-78: CUDA launch syntax, device
#      allocations) are deleted; ref_emu.cpp's ref_render runs the same three
#      kernels and the same merge sort in their order;
#   7. the `1.8l` literal in processAtomsKernel (Rasterizer.cu:221) becomes
#      `1.8`: CUDA device code has no long double and computes it in double,
#      where the host compiler would use x87 extended precision.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${LIMA_REF_ROOT:-/root/reference}"
SRC="$REF_ROOT/Quantom/Quantom"
OUT="$HERE/_ref"
if [ ! -f "$SRC/Engine.cu" ]; then
    echo "build_ref.sh: reference sources not found under $SRC; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d /tmp/lima_ref_build.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT

for f in Engine.cu Engine.cuh Bodies.cuh QuantomTypes.cuh Simulation.cuh Forcefield.cuh Filehandling.h \
         Rasterizer.cu Rasterizer.cuh; do
    cp "$SRC/$f" "$TMP/$f"
done
cp "$HERE/ref_shim/Constants.cuh" "$TMP/Constants.cuh"

# 2. NeighborList::loadData double increment
n=$(grep -cE '^[[:space:]]*i \+= blockDim\.x;[[:space:]]*$' "$TMP/Bodies.cuh" || true)
[ "$n" = "1" ] || { echo "build_ref.sh: expected one loadData increment line, found $n" >&2; exit 1; }
sed -i -E '/^[[:space:]]*i \+= blockDim\.x;[[:space:]]*$/d' "$TMP/Bodies.cuh"

# 3. drop Engine::step (from its signature to the first top-level closing brace)
n=$(grep -c '^void Engine::step() {' "$TMP/Engine.cu" || true)
[ "$n" = "1" ] || { echo "build_ref.sh: Engine::step signature not found" >&2; exit 1; }
awk 'BEGIN{skip=0} /^void Engine::step\(\) \{/{skip=1} { if(!skip) print; else if ($0 ~ /^}/) skip=0 }' \
    "$TMP/Engine.cu" > "$TMP/Engine.cu.new" && mv "$TMP/Engine.cu.new" "$TMP/Engine.cu"
! grep -q '<< <' "$TMP/Engine.cu" || { echo "build_ref.sh: launch syntax left in Engine.cu" >&2; exit 1; }

# 4. force hook at the top of integratePosition
n=$(grep -c '^__device__ void integratePosition(Float3\* pos, Float3\* pos_tsub1' "$TMP/Engine.cu" || true)
[ "$n" = "1" ] || { echo "build_ref.sh: integratePosition signature not found" >&2; exit 1; }
sed -i '/^__device__ void integratePosition(Float3\* pos, Float3\* pos_tsub1/a\	lima_ref_force_hook(p_index, force);' "$TMP/Engine.cu"

# 5. barriers at the two intra-block races (see the header)
n=$(grep -cE '^[[:space:]]*utility_buffer\[threadIdx\.x\] = Float3\((0\.f|0, 0, 0)\);[[:space:]]*$' "$TMP/Engine.cu" || true)
[ "$n" = "3" ] || { echo "build_ref.sh: expected 3 bonded accumulator resets, found $n" >&2; exit 1; }
sed -i -E '/^[[:space:]]*utility_buffer\[threadIdx\.x\] = Float3\((0\.f|0, 0, 0)\);[[:space:]]*$/a\	__syncthreads();' "$TMP/Engine.cu"
n=$(grep -c 'applyHyperpos(&compound_state.positions\[0\], &compound_state.positions\[threadIdx.x\]);.*So all particles follows p0' "$TMP/Engine.cu" || true)
[ "$n" = "1" ] || { echo "build_ref.sh: PBC hyperpos line not found" >&2; exit 1; }
sed -i '/applyHyperpos(&compound_state.positions\[0\], &compound_state.positions\[threadIdx.x\]);.*So all particles follows p0/i\	__syncthreads();' "$TMP/Engine.cu"

# 6. drop the Rasterizer member functions (signature to the first top-level closing brace)
n=$(grep -cE '^[A-Za-z]+\*? Rasterizer::(render|getAllAtoms|sortAtoms|processAtoms)\(' "$TMP/Rasterizer.cu" || true)
[ "$n" = "4" ] || { echo "build_ref.sh: expected 4 Rasterizer member functions, found $n" >&2; exit 1; }
awk 'BEGIN{skip=0} /^[A-Za-z]+\*? Rasterizer::(render|getAllAtoms|sortAtoms|processAtoms)\(/{skip=1}
     { if(!skip) print; else if ($0 ~ /^}/) skip=0 }' "$TMP/Rasterizer.cu" > "$TMP/Rasterizer.cu.new" &&
    mv "$TMP/Rasterizer.cu.new" "$TMP/Rasterizer.cu"
! grep -qE '<< ?<' "$TMP/Rasterizer.cu" || { echo "build_ref.sh: launch syntax left in Rasterizer.cu" >&2; exit 1; }

# 7. the long double literal of processAtomsKernel
n=$(grep -c ' \* 1\.8l;' "$TMP/Rasterizer.cu" || true)
[ "$n" = "1" ] || { echo "build_ref.sh: expected one 1.8l literal, found $n" >&2; exit 1; }
sed -i 's/ \* 1\.8l;/ * 1.8;/' "$TMP/Rasterizer.cu"

CXX="${CXX:-g++}"
"$CXX" -std=c++17 -O3 -march=x86-64-v3 -ffp-contract=off -fno-fast-math -pthread -fPIC -shared -w \
    -I"$TMP" -I"$HERE/ref_shim" \
    "$HERE/ref_emu.cpp" "$HERE/ref_switch.S" -o "$OUT/libref_lima.so.tmp"
mv "$OUT/libref_lima.so.tmp" "$OUT/libref_lima.so"
echo "built $OUT/libref_lima.so"
