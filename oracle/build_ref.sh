#!/bin/sh
# Test infrastructure only: compiles parts of the reference (ATLAS 3.11.41)
# from its own C sources, unmodified and where they lie, to pin the CPU
# oracle.  Nothing here is linked by the GPU library.
#
#   oracle/_ref/libatlref.so         the C reference level-3 BLAS
#                                    (src/blas/reference/level3/ATL_{d,s}ref*)
#   oracle/_ref/libatlref_lapack.so  the reference's LAPACK path
#                                    (src/lapack: getrfC/getrfR/getf2/laswp/getrs,
#                                    potrf/potrfL/potrfU/potrs, geqrf/geqrr/geqr2/
#                                    larfg/larft/larfb/larf, ilaenv/laGetB/lamch/
#                                    lapy2, src/auxil/ATL_xerbla,
#                                    interfaces/lapack/C/src/clapack_ilaenv) over
#                                    the C reference level-1/2/3 BLAS, reached
#                                    through oracle/refshim/refcblas.c
#
# The LAPACK sources include headers that ATLAS's configure / tuning steps
# write (type sizes, cache sizes, machine parameters, amm views, tuned NBs);
# oracle/refshim/include holds small hand-written stand-ins for them.  They
# set only type sizes, IEEE constants and blocking factors, so they change
# rounding (split points), not the algorithms.
#
# The reference is found at $ATLAS_REF_SRC (default: /root/reference).  When
# it is absent the recipe says so and exits 0: the committed golden vectors
# (tests/golden/) are what the tests read.
set -e
REF=${ATLAS_REF_SRC:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
CC=${CC:-gcc}
if [ ! -d "$REF/src/blas/reference/level3" ] || [ ! -d "$REF/src/lapack" ]; then
  echo "reference sources not found at $REF: oracle/_ref not built"
  exit 0
fi
mkdir -p "$OUT/obj" "$OUT/lobj"
CF="-O2 -fPIC -ffp-contract=off"

# --- reference level-3 BLAS ---------------------------------------------
OBJS=""
for p in ATL_drefgemm ATL_dreftrsm ATL_drefsyrk ATL_dreftrmm ATL_srefgemm; do
  for f in "$REF"/src/blas/reference/level3/${p}*.c; do
    o="$OUT/obj/$(basename "$f" .c).o"
    $CC $CF -I"$REF/include" -c "$f" -o "$o"
    OBJS="$OBJS $o"
  done
done
$CC -shared -o "$OUT/libatlref.so" $OBJS -lm

# --- reference LAPACK over the reference BLAS ----------------------------
INC="-I$HERE/refshim/include -I$REF/include"
LOBJS=""
lcc() {  # lcc <type macro> <source> <object name>
  $CC -D"$1" $CF $INC -c "$2" -o "$OUT/lobj/$3.o"
  LOBJS="$LOBJS $OUT/lobj/$3.o"
}
for f in getrfC getrfR getrf getf2 laswp getrs potrf potrfL potrfU potrs \
         geqrf geqrr geqr2 larfg larft larfb larf ilaenv lamch lapy2; do
  lcc DREAL "$REF/src/lapack/ATL_$f.c" "ATL_d$f"
done
for t in SREAL DREAL SCPLX DCPLX; do  # ilaenv refers to all four
  lcc $t "$REF/src/lapack/ATL_laGetB.c" "ATL_laGetB_$t"
done
lcc DREAL "$REF/src/auxil/ATL_xerbla.c" ATL_xerbla
lcc DREAL "$REF/interfaces/lapack/C/src/clapack_ilaenv.c" clapack_ilaenv
lcc DREAL "$HERE/refshim/refcblas.c" refcblas
L1="$REF/src/blas/reference/level1"
for f in "$REF"/src/blas/reference/level3/ATL_dref*.c \
         "$REF"/src/blas/reference/level2/ATL_drefgemv*.c \
         "$REF"/src/blas/reference/level2/ATL_drefger*.c \
         "$REF"/src/blas/reference/level2/ATL_dreftrsv*.c \
         "$L1/ATL_idrefamax.c" "$L1/ATL_drefscal.c" "$L1/ATL_drefswap.c" \
         "$L1/ATL_drefcopy.c" "$L1/ATL_drefdot.c" "$L1/ATL_drefnrm2.c"; do
  o="$OUT/lobj/$(basename "$f" .c).o"
  $CC $CF -I"$REF/include" -c "$f" -o "$o"
  LOBJS="$LOBJS $o"
done
$CC -shared -Wl,--no-undefined -o "$OUT/libatlref_lapack.so" $LOBJS -lm
rm -rf "$OUT/obj" "$OUT/lobj"
echo "built $OUT/libatlref.so $OUT/libatlref_lapack.so"
