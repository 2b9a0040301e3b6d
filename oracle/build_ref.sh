#!/usr/bin/env bash
# TEST INFRASTRUCTURE: compiles the UNMODIFIED origo-tlno reference engine
# from its own sources (read in place under /root/reference, never copied)
# together with oracle/ref_harness.cpp into oracle/_ref/libtlno_ref.so.
#
# The reference's CMake build is not used; this recipe compiles the few
# translation units of the integral hot path directly with g++, with the
# reference's AVX2 "Release" options (CMakeLists.txt:9-34: -march=x86-64-v3,
# -O3 -DNDEBUG, OpenMP, C++17).  Output goes only to oracle/_ref/.
#
# Usage: oracle/build_ref.sh [reference_root]
#   reference_root defaults to $TLNO_REFERENCE_ROOT, then /root/reference.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${TLNO_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
# The image may export CXX pointing at a compiler without libgomp; the
# reference build needs OpenMP, so use the system g++ unless REF_CXX is set.
CXX="${REF_CXX:-/usr/bin/g++}"
if [ ! -d "$REF/integrals" ]; then
    echo "build_ref: reference sources not found at $REF" >&2
    exit 2
fi
mkdir -p "$OBJ" "$OBJ/avx512"
FLAGS=(-std=c++17 -O3 -DNDEBUG -march=x86-64-v3 -mtune=generic -fopenmp -fPIC -I"$REF" -w)
# the reference's AVX-512 route (TLNO_SIMD=avx512: -march=x86-64-v4), built
# into oracle/_ref/libtlno_ref_avx512.so when the host compiler accepts it
FLAGS512=(-std=c++17 -O3 -DNDEBUG -march=x86-64-v4 -mtune=generic -fopenmp -fPIC -I"$REF" -w)
SRCS=(
  core/shell/shell_math.cpp
  core/shell/shell_contract.cpp
  core/shell/cart2sph.cpp
  core/math/general_math.cpp
  integrals/one_electron/onee_integrals.cpp
  integrals/one_electron/onee_matrices.cpp
  integrals/two_electron/fock/jk_direct.cpp
  core/basis/basis_general.cpp
  core/basis/get_sto3g_params.cpp
  core/basis/get_4_31g_params.cpp
  core/basis/get_6_31g_params.cpp
  core/basis/get_6_31g_d_params.cpp
  core/basis/get_6_31g_dp_params.cpp
  core/basis/get_def2_svp_params.cpp
  core/basis/get_def2_tzvp_params.cpp
  benchmarks/common/molecule_io.cpp
)
pids=()
objs=()
objs512=()
for s in "${SRCS[@]}"; do
  b="$(echo "$s" | tr '/' '_' ).o"
  objs+=("$OBJ/$b")
  objs512+=("$OBJ/avx512/$b")
  if [ ! -f "$OBJ/$b" ] || [ "$REF/$s" -nt "$OBJ/$b" ]; then
    "$CXX" "${FLAGS[@]}" -c "$REF/$s" -o "$OBJ/$b" &
    pids+=($!)
  fi
  if [ ! -f "$OBJ/avx512/$b" ] || [ "$REF/$s" -nt "$OBJ/avx512/$b" ]; then
    "$CXX" "${FLAGS512[@]}" -c "$REF/$s" -o "$OBJ/avx512/$b" &
    pids+=($!)
  fi
done
for h in ref_harness ref_frontend; do
  objs+=("$OBJ/$h.o")
  objs512+=("$OBJ/avx512/$h.o")
  if [ ! -f "$OBJ/$h.o" ] || [ "$HERE/$h.cpp" -nt "$OBJ/$h.o" ]; then
    "$CXX" "${FLAGS[@]}" -c "$HERE/$h.cpp" -o "$OBJ/$h.o" &
    pids+=($!)
  fi
  if [ ! -f "$OBJ/avx512/$h.o" ] || [ "$HERE/$h.cpp" -nt "$OBJ/avx512/$h.o" ]; then
    "$CXX" "${FLAGS512[@]}" -c "$HERE/$h.cpp" -o "$OBJ/avx512/$h.o" &
    pids+=($!)
  fi
done
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -shared -fopenmp -o "$OUT/libtlno_ref.so" "${objs[@]}"
echo "build_ref: wrote $OUT/libtlno_ref.so"
"$CXX" -shared -fopenmp -o "$OUT/libtlno_ref_avx512.so" "${objs512[@]}"
echo "build_ref: wrote $OUT/libtlno_ref_avx512.so"
# The C++ shim test (tests/shim/shim_test.cpp) compiled against the
# reference's headers, linking the compiled reference and the engine library
# (built before this script runs).
ROOT="$(cd "$HERE/.." && pwd)"
GPU_LIB="$ROOT/origo_tlno_b200/_lib"
if [ -f "$GPU_LIB/libtlno_gpu.so" ]; then
  "$CXX" -std=c++17 -O2 -fopenmp -I"$REF" -I"$ROOT" -w "$ROOT/tests/shim/shim_test.cpp" -o "$OUT/shim_test" \
    -L"$OUT" -ltlno_ref -L"$GPU_LIB" -ltlno_gpu -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../origo_tlno_b200/_lib'
  echo "build_ref: wrote $OUT/shim_test"
fi
