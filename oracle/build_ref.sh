#!/usr/bin/env bash
# Compiles the UNMODIFIED reference C++ engine (monoprop) from its own sources, plus the stand-in
# headers/stubs in oracle/ref_shim and oracle/ref_stubs.cpp and the C-ABI driver oracle/ref_driver.cpp,
# into oracle/_ref/. The reference tree is only read; nothing is copied into this repository.
#
# Three builds of the same sources, differing only in the instruction set:
#   libmpref.so      -march=x86-64-v3 (AVX2/FMA/BMI2): runs on any host CPU of the GPU machines; the oracle
#                    the tests use;
#   libmpref_v4.so   -march=x86-64-v4 (adds AVX-512F/BW/CD/DQ/VL);
#   libmpref_spr.so  -march=sapphirerapids: what the reference's own default build (-march=native,
#                    cmake/compiler_flags/CXXFlags.cmake) selects on the GPU machines' Sapphire Rapids hosts.
# The timing arm runs the build matching the host CPU's extensions (the reference's stock flags there).
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default: $MONOPROP_REFERENCE, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${MONOPROP_REFERENCE:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/cpp/monoprop" ]; then
    echo "reference sources not found under $REF; oracle/_ref not rebuilt" >&2
    exit 0
fi
CXX="${CXX:-g++}"
SRCS=("$REF/cpp/monoprop/Evolution.cpp" "$REF/cpp/monoprop/MPFunctions.cpp" "$REF/cpp/monoprop/MPGraph.cpp"
      "$REF/cpp/monoprop/Validation.cpp" "$REF/cpp/monoprop/detail/graph_encoding/MPGraphEncoding.cpp"
      "$REF/cpp/monoprop/detail/pare/PareGraph.cpp" "$REF/cpp/monoprop/detail/mpi/MPICompat.cpp"
      "$HERE/ref_stubs.cpp" "$HERE/ref_driver.cpp")
build_variant() { # $1 = -march value, $2 = object dir, $3 = library name
    local march="$1" objdir="$OUT/$2" lib="$OUT/$3"
    local flags=(-std=c++23 -O3 "-march=$march" -DNDEBUG -fPIC -pthread -w
                 -I "$HERE/ref_shim" -I "$REF/cpp/include" -I "$REF/cpp")
    mkdir -p "$objdir"
    local pids=() objs=()
    for s in "${SRCS[@]}"; do
        local o="$objdir/$(basename "${s%.cpp}").o"
        objs+=("$o")
        if [ ! -f "$o" ] || [ "$s" -nt "$o" ]; then
            "$CXX" "${flags[@]}" -c "$s" -o "$o" &
            pids+=($!)
        fi
    done
    for p in "${pids[@]}"; do wait "$p"; done
    if [ ! -f "$lib" ] || [ -n "$(find "${objs[@]}" -newer "$lib")" ]; then
        "$CXX" -shared -pthread -o "$lib" "${objs[@]}"
    fi
    echo "built $lib"
}
build_variant x86-64-v3 obj libmpref.so
build_variant x86-64-v4 obj_v4 libmpref_v4.so
build_variant sapphirerapids obj_spr libmpref_spr.so
