#!/usr/bin/env bash
# Build recipe for the unmodified CosTuuM reference (test infrastructure only).
#
# Compiles, from the reference sources where they lie (nothing is copied into
# this repository), into oracle/_ref/:
#   * CosTuuM<ext-suffix>.so  -- the reference's own CPython module
#                               (src/CTMModule.cpp), used to make golden
#                               fixtures and as the timed CPU baseline;
#   * libref_driver.so       -- oracle/ref_driver.cpp, a C-ABI harness that
#                               instantiates the reference's task objects
#                               (TMatrixM0Task chains, TMatrixMAllTask, ...)
#                               and runs them under the reference's QuickSched.
#
# The reference's CMake does not configure in this image (CMake 4 rejects its
# cmake_minimum_required and the missing .git breaks its version parsing), so
# the two generated headers are written here by sed, as its CMake would.
#
# Usage: oracle/build_ref.sh [--optional] [REFERENCE_ROOT]
#        (REFERENCE_ROOT defaults to $COSTUUM_REFERENCE; --optional: exit 0
#        when neither names a reference source tree)
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OPTIONAL=0
if [ "${1:-}" = "--optional" ]; then
  OPTIONAL=1
  shift
fi
REF="${1:-${COSTUUM_REFERENCE:-}}"
OUT="$HERE/_ref"
GEN="$OUT/gen"

if [ -z "$REF" ] || [ ! -f "$REF/src/CTMModule.cpp" ]; then
  if [ "$OPTIONAL" = 1 ]; then
    exit 0
  fi
  echo "build_ref.sh: reference sources not found under $REF" >&2
  exit 1
fi

mkdir -p "$GEN"

# generated headers: Release configuration, OpenMP + POSIX, double precision
sed -e 's/#cmakedefine HAVE_ASSERTIONS/\/\* HAVE_ASSERTIONS off \*\//' \
    -e 's/#cmakedefine HAVE_OPENMP/#define HAVE_OPENMP/' \
    -e 's/#cmakedefine HAVE_POSIX/#define HAVE_POSIX/' \
    -e 's/#cmakedefine HAVE_WINDOWS/\/\* HAVE_WINDOWS off \*\//' \
    -e 's/#cmakedefine HAVE_MULTIPRECISION/\/\* HAVE_MULTIPRECISION off \*\//' \
    -e 's/#cmakedefine HAVE_QUAD_PRECISION/\/\* HAVE_QUAD_PRECISION off \*\//' \
    -e 's/@MAX_NUM_THREADS@/256/' \
    "$REF/src/Configuration.hpp.in" > "$GEN/Configuration.hpp"
sed -e "s|@DRAINEDUSTPROPERTIESDATALOCATION@|$REF/data/|" \
    "$REF/src/DraineDustPropertiesDataLocation.hpp.in" \
    > "$GEN/DraineDustPropertiesDataLocation.hpp"

# QuickSched (C), position independent so it can go into shared objects
for f in qsched queue; do
  gcc -O2 -fPIC -fopenmp -I "$REF/quicksched" -c "$REF/quicksched/$f.c" \
      -o "$OUT/$f.o"
done

PYINC="$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["include"])')"
NPINC="$(python3 -c 'import numpy; print(numpy.get_include())')"
EXT="$(python3 -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
CXXFLAGS=(-O3 -std=c++11 -fPIC -fopenmp -w -I "$GEN" -I "$REF/src"
          -I "$REF/quicksched")

# the reference's Python module
g++ "${CXXFLAGS[@]}" -shared -I "$PYINC" -I "$NPINC" \
    "$REF/src/CTMModule.cpp" "$OUT/qsched.o" "$OUT/queue.o" \
    -o "$OUT/CosTuuM$EXT"

# the task-level C-ABI harness
g++ "${CXXFLAGS[@]}" -shared "$HERE/ref_driver.cpp" \
    "$OUT/qsched.o" "$OUT/queue.o" -o "$OUT/libref_driver.so"

echo "build_ref.sh: built $OUT/CosTuuM$EXT and $OUT/libref_driver.so"
