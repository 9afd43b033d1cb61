#!/bin/sh
# Compile the reference's own CPU sources (double precision, long ints,
# OpenMP) into oracle/_ref/libgrid_ref.so, linked against the project's
# FFTW stand-in (oracle/shim).  Reads the sources where they lie; writes only
# under oracle/_ref/.  Mirrors the reference build's configuration
# (make.conf:45,73-97 for REAL=double, INT=long; src/Makefile:18-19,96-104 for
# git-version.h and proto.h) without running the reference's build system.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or set LIBGRID_REFERENCE)
set -eu
REF=${1:-${LIBGRID_REFERENCE:-}}
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh REFERENCE_ROOT (or set LIBGRID_REFERENCE)" >&2
  exit 2
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
GEN="$OUT/gen"
SRC="$REF/src"

if [ ! -d "$SRC" ]; then
  echo "build_ref.sh: reference sources not found at $SRC" >&2
  exit 1
fi
mkdir -p "$GEN" "$OUT/obj"

# proto.h: exported prototypes, CUDA entries dropped (non-CUDA build).
grep -h '^EXPORT' "$SRC"/*.c "$SRC"/ext-cuda/func*.c | tr '{' ';' | sed -e 's/EXPORT //g' \
  | grep -v cuda > "$GEN/proto.h"
echo '#define VERSION "reference-oracle-build"' > "$GEN/git-version.h"

DTYPE="-DREAL=double -DDOUBLE_PREC -DCREAL=creal -DCIMAG=cimag -DCONJ=conj -DPOW=pow -DSQRT=sqrt -DCSQRT=csqrt -DEXP=exp -DCEXP=cexp -DLOG=log -DCLOG=clog -DCOS=cos -DSIN=sin -DTAN=tan -DATAN2=atan2 -DFABS=fabs -DCABS=cabs -DACOS=acos -DASIN=asin -DATAN=atan -DTANH=tanh -DCOSH=cosh -DSINH=sinh -DCPOW=cpow -DCARG=carg -DINT=long -DLONG_INT -DABS=labs"
CFLAGS="-std=gnu89 -O2 -fPIC -fopenmp -ffp-contract=off -w -DHBAR=1.0 $DTYPE -I$GEN -I$HERE/shim -I$SRC"

FILES="cgrid.c cgrid_fft.c cgrid_diff.c rgrid.c rgrid_fft.c rgrid_diff.c ngrid.c grid_wf.c grid_wf_fft.c grid_wf_diag.c grid_wf_cn.c cgrid_bc.c rgrid_bc.c threads.c linalg.c ctimer.c interpolate.c grid_fft.c grid_wf_analyze.c rand.c rgrid_func.c"
OBJS=""
for f in $FILES; do
  o="$OUT/obj/${f%.c}.o"
  gcc $CFLAGS -c "$SRC/$f" -o "$o"
  OBJS="$OBJS $o"
done
gcc -std=gnu99 -O2 -fPIC -fopenmp -I"$HERE/shim" -c "$HERE/shim/fftw_shim.c" -o "$OUT/obj/fftw_shim.o"
gcc -std=gnu99 -O2 -fPIC -fopenmp -c "$HERE/gbo_fft.c" -o "$OUT/obj/gbo_fft.o"
gcc -shared -fopenmp -o "$OUT/libgrid_ref.so" $OBJS "$OUT/obj/fftw_shim.o" "$OUT/obj/gbo_fft.o" -lm
echo "built $OUT/libgrid_ref.so"
