#!/usr/bin/env bash
# build_ref.sh -- compile the reference's own CPU code from its read-only
# sources into oracle/_ref/ (git-ignored; the built files travel with the
# repository snapshot to the GPU box, where the sources are absent).
#
# Built (direct compiler commands; the reference's CMake is not used because
# it requires GMP headers that this image lacks):
#   _ref/cpu_goldbach   src/cpu_goldbach.cpp + src/segmented_sieve.cpp
#   _ref/test_sieve     src/test_sieve.cpp + src/segmented_sieve.cpp
#   _ref/test_bitset    src/test_bitset.cpp + src/prime_bitset.cpp (OpenMP)
#   _ref/libgbref.so    oracle/ref_shim.cpp + src/segmented_sieve.cpp +
#                       src/cpu_goldbach.cpp (main renamed)
#   _ref/libgbref_p2.so oracle/ref_phase2_shim.cu, which includes
#                       src/goldbach.cu (main renamed) + src/prime_bitset.cpp
#   _ref/goldbach       src/goldbach.cu + src/prime_bitset.cpp as they are, for
#                       sm_100a: the reference's own GPU range verifier, used
#                       only to time it on the same B200 (its tiled sieve has
#                       an unsynchronised shared-memory update, so it is not a
#                       checker)
# Flags are portable (-O3, no -march=native) so the binaries run on any
# x86-64 host.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference checkout: GB_REFERENCE_DIR, else a sibling of the repository
REF="${GB_REFERENCE_DIR:-$HERE/../../reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "build_ref.sh: reference sources not found at $REF; keeping prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX=g++
NVCC="${NVCC:-nvcc}"
CXXFLAGS="-O3 -std=c++17"
S="$REF/src"
I="$REF/include"

$CXX $CXXFLAGS "$S/cpu_goldbach.cpp" "$S/segmented_sieve.cpp" -o "$OUT/cpu_goldbach"
$CXX $CXXFLAGS "$S/test_sieve.cpp" "$S/segmented_sieve.cpp" -o "$OUT/test_sieve"
$CXX $CXXFLAGS -fopenmp -I"$I" "$S/test_bitset.cpp" "$S/prime_bitset.cpp" -o "$OUT/test_bitset"

# libgbref.so: objects compiled one by one so that only cpu_goldbach.cpp
# sees the main() rename.
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
$CXX $CXXFLAGS -fPIC -c "$S/segmented_sieve.cpp" -o "$TMP/segmented_sieve.o"
$CXX $CXXFLAGS -fPIC -Dmain=gbref_cpu_goldbach_main -c "$S/cpu_goldbach.cpp" -o "$TMP/cpu_goldbach.o"
$CXX $CXXFLAGS -fPIC -c "$HERE/ref_shim.cpp" -o "$TMP/ref_shim.o"
$CXX -shared -o "$OUT/libgbref.so" "$TMP/ref_shim.o" "$TMP/segmented_sieve.o" "$TMP/cpu_goldbach.o" -lpthread

# libgbref_p2.so: the reference's Phase-2 host helpers (static in goldbach.cu).
$CXX $CXXFLAGS -fPIC -fopenmp -I"$I" -c "$S/prime_bitset.cpp" -o "$TMP/prime_bitset.o"
$NVCC -O3 -std=c++17 -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a \
  -I"$S" -I"$I" -c "$HERE/ref_phase2_shim.cu" -o "$TMP/ref_phase2_shim.o"
$NVCC -shared -cudart static -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp -o "$OUT/libgbref_p2.so" \
  "$TMP/ref_phase2_shim.o" "$TMP/prime_bitset.o"
# the reference GPU verifier, unmodified (its CMake flags: -O3, OpenMP)
$NVCC -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp,-O3 \
  -I"$I" "$S/goldbach.cu" "$S/prime_bitset.cpp" -o "$OUT/goldbach" -lgomp -lpthread
echo "build_ref.sh: built $(ls "$OUT" | tr '\n' ' ')"
