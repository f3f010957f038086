#!/usr/bin/env bash
# Builds oracle/_ref/libshape_dropin.so: the calc_fits drop-in
# (shape-cuda-v1.2_b200/dropin/shape_b200_dropin.c) and the plane-of-sky
# drop-ins (dropin/shape_b200_pos.c) compiled against the
# reference's headers, as a maintainer would compile it inside the reference
# tree, plus a small test harness (oracle/dropin_harness.c). The drop-in's
# entry points are renamed (-DSHAPE_B200_CALC_FITS=...) so that tests can run
# it beside the reference's own calc_fits in one process. Links against
# oracle/_ref/libshape_ref.so (oracle/build_ref.sh) and the engine library.
# Test infrastructure only.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/.." && pwd)"
REF_ROOT="${REF_ROOT:-$(cd "$REPO/.." && pwd)/reference}"
SRC="$REF_ROOT/src"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
LIBDIR="$REPO/shape-cuda-v1.2_b200/lib"
CC="${CC:-gcc}"
CFLAGS="-O2 -ffp-contract=off -fPIC -w -std=gnu99"
if [ ! -d "$SRC/shape" ]; then
    echo "build_dropin.sh: reference headers not found under $SRC" >&2
    exit 2
fi
if [ ! -f "$OUT/libshape_ref.so" ] || [ ! -f "$LIBDIR/libshape_b200.so" ]; then
    echo "build_dropin.sh: build oracle/_ref/libshape_ref.so and the engine library first" >&2
    exit 2
fi
mkdir -p "$OBJ"
INC="-I$SRC/shape -I$SRC/util -I$SRC/nr -I$SRC/astro -I$SRC/pgm -I$SRC/HostMultiThreading -I/usr/local/cuda/include -I$REPO/include -I$REPO/shape-cuda-v1.2_b200/dropin -I$HERE"
$CC $CFLAGS -c -I- -I"$HERE/refshim/shape" $INC \
    -DSHAPE_B200_CALC_FITS=calc_fits_b200dropin -DSHAPE_B200_CALC_FITS_CHI2=calc_fits_chi2_b200dropin \
    "$REPO/shape-cuda-v1.2_b200/dropin/shape_b200_dropin.c" -o "$OBJ/dropin.o"
$CC $CFLAGS -c -I- -I"$HERE/refshim/shape" $INC -DSHAPE_B200_POS_PREFIX=b200dropin_ \
    "$REPO/shape-cuda-v1.2_b200/dropin/shape_b200_pos.c" -o "$OBJ/dropin_pos.o"
$CC $CFLAGS -c -I- -I"$HERE/refshim/shape" $INC "$HERE/dropin_harness.c" -o "$OBJ/dropin_harness.o"
$CC -shared -o "$OUT/libshape_dropin.so" "$OBJ/dropin.o" "$OBJ/dropin_pos.o" "$OBJ/dropin_harness.o" \
    -L"$OUT" -lshape_ref -L"$LIBDIR" -lshape_b200 -lm \
    -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../shape-cuda-v1.2_b200/lib' -Wl,--no-undefined
echo "built $OUT/libshape_dropin.so"
