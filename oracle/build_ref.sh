#!/usr/bin/env bash
# Builds the reference's own CPU gridder/degridder (DDFacet's pybind11 module
# _pyGridderSmearPols3x) from its four C++ sources, in place under the
# read-only reference checkout, into oracle/_ref/.  Test infrastructure only:
# the module is the parity checker and the timed CPU baseline, never product.
#
# Flags follow DDFacet/Gridder/CMakeLists.txt:5-25 (-O3 -ffast-math -fopenmp
# -std=c++14) except -march=native, which is left out so the .so also runs on
# a host CPU other than the one that built it.
set -euo pipefail
REF=${DDFACET_REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/DDFacet/Gridder"
if [ ! -d "$SRC" ]; then
  echo "build_ref: reference sources not found at $SRC" >&2
  exit 1
fi
mkdir -p "$OUT"
PY=${PYTHON:-python}
PYINC=$($PY -c 'import sysconfig;print(sysconfig.get_paths()["include"])')
NPINC=$($PY -c 'import numpy;print(numpy.get_include())')
PBINC=$($PY -c 'import pybind11;print(pybind11.get_include())')
EXT=$($PY -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')
TARGET="$OUT/_pyGridderSmearPols3x$EXT"
if [ -f "$TARGET" ] && [ "${FORCE:-0}" != "1" ]; then
  echo "build_ref: $TARGET up to date"
  exit 0
fi
g++ -O3 -ffast-math -fopenmp -std=c++14 -shared -fPIC \
  -DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION \
  -I"$PYINC" -I"$NPINC" -I"$NPINC/numpy" -I"$PBINC" -I"$SRC" \
  "$SRC/GridderSmearPols.cc" "$SRC/Semaphores.cc" "$SRC/JonesServer.cc" \
  "$SRC/DecorrelationHelper.cc" -o "$TARGET" -lrt
echo "build_ref: built $TARGET"
