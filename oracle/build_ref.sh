#!/bin/sh
# Compiles the parts of the reference's accelsearch path that build from the
# reference's own source files with no external library, into oracle/_ref/.
# src/fresnl.c (Cephes Fresnel integrals, used by gen_z_response at
# src/responses.c:291-292) qualifies as is.  src/output.c (nice_output_1 /
# nice_output_2, the value(error) format of the ACCEL text file) needs only
# FFTW's type names through include/presto.h, which refshim/fftw3.h declares;
# the library exports just those two functions, and --gc-sections drops the
# file's other functions with their references to the rest of libpresto.
# Every other hot-path file calls FFTW, GSL or glib, none of which exist here.
# Nothing from the reference is copied into the repository; the objects land
# in oracle/_ref/, which git ignores.
set -e
REF=${PRESTO_REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/src/fresnl.c" ]; then
    echo "build_ref.sh: reference tree not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
$( [ -x /usr/bin/gcc ] && echo /usr/bin/gcc || echo gcc ) -O2 -g -fPIC -shared -o "$OUT/libref_fresnl.so" "$REF/src/fresnl.c" -lm
echo "built $OUT/libref_fresnl.so from $REF/src/fresnl.c"
CC=$( [ -x /usr/bin/gcc ] && echo /usr/bin/gcc || echo gcc )
echo 'REF { global: nice_output_1; nice_output_2; local: *; };' > "$OUT/output.map"
$CC -O2 -g -fPIC -ffunction-sections -fdata-sections -I "$HERE/refshim" -I "$REF/include" \
    -c "$REF/src/output.c" -o "$OUT/output.o"
$CC -shared -Wl,--gc-sections -Wl,--version-script="$OUT/output.map" -o "$OUT/libref_output.so" \
    "$OUT/output.o" -lm
echo "built $OUT/libref_output.so from $REF/src/output.c"
# The polishing interpolators and candidate properties: src/characteristics.c
# (calc_props, calc_rzwerrs, get_localpower3d, get_derivs3d), src/rzinterp.c,
# src/rzwinterp.c, src/responses.c, src/fresnl.c and src/vectors.c, unmodified,
# linked with refshim/refshim.c (malloc-backed fftwf_malloc/free and an FP64
# forward realfft standing in for FFTW).
cat > "$OUT/polish.map" <<'MAP'
REF { global: calc_props; calc_rzwerrs; get_localpower3d; get_derivs3d; rz_interp;
      rzw_interp; gen_r_response; gen_z_response; gen_w_response; r_resp_halfwidth;
      z_resp_halfwidth; w_resp_halfwidth; vect_free; local: *; };
MAP
POBJ=""
for f in characteristics rzinterp rzwinterp responses fresnl vectors; do
    $CC -O2 -g -fPIC -ffunction-sections -fdata-sections -I "$HERE/refshim" -I "$REF/include" \
        -c "$REF/src/$f.c" -o "$OUT/p_$f.o"
    POBJ="$POBJ $OUT/p_$f.o"
done
$CC -O2 -g -fPIC -c "$HERE/refshim/refshim.c" -o "$OUT/p_refshim.o"
$CC -shared -Wl,--gc-sections -Wl,--version-script="$OUT/polish.map" -Wl,-z,defs \
    -o "$OUT/libref_polish.so" $POBJ "$OUT/p_refshim.o" -lm
echo "built $OUT/libref_polish.so from $REF/src/{characteristics,rzinterp,rzwinterp,responses,fresnl,vectors}.c"
