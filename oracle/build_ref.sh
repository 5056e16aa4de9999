#!/usr/bin/env bash
# Compiles the UNMODIFIED reference C++ engine (monoprop) from its own sources, plus the stand-in
# headers/stubs in oracle/ref_shim and oracle/ref_stubs.cpp and the C-ABI driver oracle/ref_driver.cpp,
# into oracle/_ref/libmpref.so. The reference tree is only read; nothing is copied into this repository.
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/cpp/monoprop" ]; then
    echo "reference sources not found under $REF; oracle/_ref not rebuilt" >&2
    exit 0
fi
mkdir -p "$OUT/obj"
CXX="${CXX:-g++}"
# x86-64-v3 (AVX2/FMA/BMI2) instead of -march=native so the library also runs on the GPU hosts' CPUs.
FLAGS=(-std=c++23 -O3 -march=x86-64-v3 -DNDEBUG -fPIC -pthread -w
       -I "$HERE/ref_shim" -I "$REF/cpp/include" -I "$REF/cpp")
SRCS=("$REF/cpp/monoprop/Evolution.cpp" "$REF/cpp/monoprop/MPFunctions.cpp" "$REF/cpp/monoprop/MPGraph.cpp"
      "$REF/cpp/monoprop/Validation.cpp" "$REF/cpp/monoprop/detail/graph_encoding/MPGraphEncoding.cpp"
      "$REF/cpp/monoprop/detail/pare/PareGraph.cpp" "$REF/cpp/monoprop/detail/mpi/MPICompat.cpp"
      "$HERE/ref_stubs.cpp" "$HERE/ref_driver.cpp")
pids=()
objs=()
for s in "${SRCS[@]}"; do
    o="$OUT/obj/$(basename "${s%.cpp}").o"
    objs+=("$o")
    if [ ! -f "$o" ] || [ "$s" -nt "$o" ]; then
        "$CXX" "${FLAGS[@]}" -c "$s" -o "$o" &
        pids+=($!)
    fi
done
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -shared -pthread -o "$OUT/libmpref.so" "${objs[@]}"
echo "built $OUT/libmpref.so"
