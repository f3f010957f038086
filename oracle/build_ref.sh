#!/usr/bin/env bash
# Builds the reference SHAPE CPU code into oracle/_ref/libshape_ref.so
# (test infrastructure: the checker and the CPU baseline, never the product).
#
# The reference's C sources are compiled where they lie under the reference
# tree (REF_ROOT; by default the reference checkout beside this repository,
# ../reference); nothing is copied. Each source is
# compiled with -I- so that its own directory is not searched for quoted
# includes, which lets oracle/refshim/shape/head.h stand in for the
# reference's head.h (that one includes an absent cfitsio by absolute path and
# a missing HybridCode directory). The CUDA port (src/CudaCode, src/CudaPR,
# src/CudaUtils, src/DebugCode) and main() (src/shape/shape-cuda-v1.0.c) are
# not compiled. Flags match the oracle restatement: -O2 -ffp-contract=off,
# no -march, so that neither side contracts FMAs.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/.." && pwd)"
REF_ROOT="${REF_ROOT:-$(cd "$REPO/.." && pwd)/reference}"
SRC="$REF_ROOT/src"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
CC="${CC:-gcc}"
CFLAGS="-O2 -ffp-contract=off -fPIC -w"
if [ ! -d "$SRC/shape" ]; then
    echo "build_ref.sh: reference sources not found under $SRC" >&2
    exit 2
fi
mkdir -p "$OBJ"
INC="-I$SRC/shape -I$SRC/util -I$SRC/nr -I$SRC/astro -I$SRC/pgm -I$SRC/HostMultiThreading -I/usr/local/cuda/include -I$REPO/include -I$HERE"
objs=()
for d in shape util nr astro pgm HostMultiThreading; do
    for f in "$SRC/$d"/*.c; do
        b="$(basename "$f" .c)"
        [ "$b" = "shape-cuda-v1.0" ] && continue
        o="$OBJ/${d}_${b}.o"
        if [ ! -f "$o" ] || [ "$f" -nt "$o" ] || [ "$HERE/refshim/shape/head.h" -nt "$o" ]; then
            $CC $CFLAGS -c -I- -I"$HERE/refshim/shape" -I"$SRC/$d" $INC "$f" -o "$o" 2>/dev/null
        fi
        objs+=("$o")
    done
done
$CC $CFLAGS -c "$HERE/refstubs.c" -o "$OBJ/refstubs.o"
$CC $CFLAGS -c -I- -I"$HERE/refshim/shape" $INC "$HERE/ref_harness.c" -o "$OBJ/ref_harness.o" 2>&1 | grep -v "obsolete option" || true
$CC -shared -o "$OUT/libshape_ref.so" "${objs[@]}" "$OBJ/refstubs.o" "$OBJ/ref_harness.o" \
    -lm -lpthread -Wl,-soname,libshape_ref.so -Wl,--no-undefined
echo "built $OUT/libshape_ref.so"
