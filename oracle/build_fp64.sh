#!/usr/bin/env bash
# Builds the FP64 restatement of the gridder/degridder (test infrastructure) into oracle/_build/.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
OUT="$HERE/_build/libddfg_fp64.so"
if [ -f "$OUT" ] && [ "$OUT" -nt "$HERE/gridder_fp64.c" ] && [ "${FORCE:-0}" != "1" ]; then exit 0; fi
gcc -O2 -std=c11 -fopenmp -fPIC -shared -Wall -o "$OUT.tmp" "$HERE/gridder_fp64.c" -lm
mv "$OUT.tmp" "$OUT"
echo "build_fp64: built $OUT"
