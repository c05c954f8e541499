#!/bin/sh
# Compiles the reference's own C reference level-3 BLAS (unmodified, from
# where the sources lie) into oracle/_ref/libatlref.so.  Used only to pin the
# oracle's BLAS restatement and as the timed CPU baseline for BLAS calls.
# Those files need only the reference's static headers; its LAPACK files need
# atlas_type.h, which only ATLAS's configure step generates, so they are not
# built here.
set -e
REF=${ATLAS_REF_SRC:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -d "$REF/src/blas/reference/level3" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OUT/obj"
SRCS=""
for p in ATL_drefgemm ATL_dreftrsm ATL_drefsyrk ATL_dreftrmm ATL_srefgemm; do
  for f in "$REF"/src/blas/reference/level3/${p}*.c; do SRCS="$SRCS $f"; done
done
OBJS=""
for f in $SRCS; do
  o="$OUT/obj/$(basename "$f" .c).o"
  ${CC:-gcc} -O2 -fPIC -ffp-contract=off -I"$REF/include" -c "$f" -o "$o"
  OBJS="$OBJS $o"
done
${CC:-gcc} -shared -o "$OUT/libatlref.so" $OBJS -lm
rm -rf "$OUT/obj"
echo "built $OUT/libatlref.so"
