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
# The accelsearch program itself: src/accelsearch.c, its command-line parser
# and the libpresto files it links (src/meson.build:56-58, -DUSEMMAP, with
# the project-wide -DUSE_FFTW_MALLOC), unmodified, linked against stand-ins of
# our own for the third-party libraries that are not in this image
# (refshim/refshim_fftw.c: FFTW's plans over an FP64 mixed-radix transform;
# refshim_glib.c: GSList; refshim_gsl.c: CDFs from oracle/accel_oracle.c,
# median, vectors, nmsimplex2, MT19937; refshim_erfa.c: angle conversions).
# oracle/_ref/accelsearch runs like the installed program (telescope "None
# (Artificial Data Set)" .inf files).
# libref_polish.so exports the polishing primitives, responses and candidate
# properties from the same objects.
OBJ="$OUT/obj"
mkdir -p "$OBJ"
PRESTO_SRC="accelsearch accelsearch_cmd accel_utils zapping characteristics responses fresnl
    vectors corr_prep corr_routines correlations fftcalls fastffts median misc_utils ioinf
    chkio maximize_rz maximize_rzw rzinterp rzwinterp output birdzap datadir database read_fft
    transpose sorter"
AOBJ=""
for f in $PRESTO_SRC; do
    $CC -O2 -g -fPIC -fopenmp -ffunction-sections -fdata-sections -DUSEMMAP -DUSE_FFTW_MALLOC \
        -DPRESTO_DATADIR='"/nonexistent"' -w -I "$HERE/refshim" -I "$REF/include" \
        -c "$REF/src/$f.c" -o "$OBJ/$f.o"
    AOBJ="$AOBJ $OBJ/$f.o"
done
SOBJ=""
for f in refshim_fftw refshim_glib refshim_gsl refshim_erfa; do
    $CC -O2 -g -fPIC -ffunction-sections -fdata-sections -I "$HERE/refshim" \
        -c "$HERE/refshim/$f.c" -o "$OBJ/$f.o"
    SOBJ="$SOBJ $OBJ/$f.o"
done
$CC -O2 -g -fPIC -ffunction-sections -fdata-sections -DORC_REAL=double \
    -c "$HERE/accel_oracle.c" -o "$OBJ/orc_stats.o"
$CC -fopenmp -Wl,--gc-sections -o "$OUT/accelsearch" $AOBJ $SOBJ "$OBJ/orc_stats.o" -lm
echo "built $OUT/accelsearch from $REF/src/accelsearch.c and the libpresto sources it links"
cat > "$OUT/polish.map" <<'MAP'
REF { global: calc_props; calc_rzwerrs; get_localpower3d; get_derivs3d; rz_interp;
      rzw_interp; gen_r_response; gen_z_response; gen_w_response; r_resp_halfwidth;
      z_resp_halfwidth; w_resp_halfwidth; vect_free; local: *; };
MAP
POBJ=""
for f in characteristics rzinterp rzwinterp responses fresnl vectors fastffts fftcalls misc_utils \
         datadir chkio transpose; do
    POBJ="$POBJ $OBJ/$f.o"
done
$CC -shared -fopenmp -Wl,--gc-sections -Wl,--version-script="$OUT/polish.map" -Wl,-z,defs \
    -o "$OUT/libref_polish.so" $POBJ $SOBJ "$OBJ/orc_stats.o" -lm
echo "built $OUT/libref_polish.so from the same objects"
# oracle/refdrv.c over the same objects (all but the program's main): the
# reference's own create_accelobs / create_subharminfos / subharm_fderivs_vol
# for plane-level checks
echo 'REF { global: refdrv_open; refdrv_close; refdrv_geometry; refdrv_plane; local: *; };' \
    > "$OUT/accel.map"
$CC -O2 -g -fPIC -fopenmp -ffunction-sections -fdata-sections -DUSEMMAP -DUSE_FFTW_MALLOC \
    -w -I "$HERE/refshim" -I "$REF/include" -c "$HERE/refdrv.c" -o "$OBJ/refdrv.o"
LOBJ=""
for f in $PRESTO_SRC; do
    [ "$f" = accelsearch ] || LOBJ="$LOBJ $OBJ/$f.o"
done
$CC -shared -fopenmp -Wl,--gc-sections -Wl,--version-script="$OUT/accel.map" -Wl,-z,defs \
    -o "$OUT/libref_accel.so" "$OBJ/refdrv.o" $LOBJ $SOBJ "$OBJ/orc_stats.o" -lm
echo "built $OUT/libref_accel.so (oracle/refdrv.c over the reference objects)"
# birdie zapping (src/zapping.c zapbirds, src/birdzap.c get_birdies) over
# the same objects, with the stand-in's MT19937
echo 'REF { global: zapbirds; get_birdies; local: *; };' > "$OUT/zap.map"
$CC -shared -fopenmp -Wl,--gc-sections -Wl,--version-script="$OUT/zap.map" -Wl,-z,defs \
    -o "$OUT/libref_zap.so" $LOBJ $SOBJ "$OBJ/orc_stats.o" -lm
echo "built $OUT/libref_zap.so (zapbirds, get_birdies)"
# The same program linked the way an installed PRESTO is (src/meson.build: a
# shared libpresto): libpresto_ref.so holds the libpresto objects with the
# stand-ins, accelsearch_dyn links against it, and accelsearch_b200 is the
# same unmodified accelsearch.o linked against presto_b200/libaccel_dropin.so
# ahead of libpresto_ref.so, so that the dynamic linker binds the main
# loop's accel.h calls (create_subharminfos, subharm_fderivs_vol,
# add_ffdotpows, search_ffdotpows, ...) to the B200 engine and everything
# else to the reference's own code.  accelsearch_dyn with
# LD_PRELOAD=presto_b200/libaccel_dropin.so does the same to the stock link.
# exported: what accelsearch.o imports, plus the list functions and the
# accelcand destructor that the drop-in library calls back into
{
    printf 'REF { global: g_slist_alloc; g_slist_remove_link; g_slist_free_1; free_accelcand;\n'
    nm -u "$OBJ/accelsearch.o" | awk '{ printf "  %s;\n", $2 }'
    printf 'local: *; };\n'
} > "$OUT/presto.map"
$CC -shared -fopenmp -Wl,--gc-sections -Wl,--version-script="$OUT/presto.map" -Wl,-z,defs \
    -o "$OUT/libpresto_ref.so" $LOBJ $SOBJ "$OBJ/orc_stats.o" -lm
$CC -fopenmp -o "$OUT/accelsearch_dyn" "$OBJ/accelsearch.o" -L"$OUT" -lpresto_ref \
    -Wl,-rpath,"\$ORIGIN" -lm
echo "built $OUT/accelsearch_dyn (src/accelsearch.c over libpresto_ref.so)"
DROPIN="$HERE/../presto_b200/libaccel_dropin.so"
if [ -f "$DROPIN" ]; then
    $CC -fopenmp -o "$OUT/accelsearch_b200" "$OBJ/accelsearch.o" \
        -L"$HERE/../presto_b200" -laccel_dropin -L"$OUT" -lpresto_ref \
        -Wl,-rpath,"\$ORIGIN" -Wl,-rpath,"\$ORIGIN/../../presto_b200" -lm
    echo "built $OUT/accelsearch_b200 (src/accelsearch.c over libaccel_dropin.so, then libpresto_ref.so)"
else
    echo "build_ref.sh: $DROPIN not built; skipping accelsearch_b200" >&2
fi
# member offsets of the structures crossing the accel.h boundary, from the
# reference's own header (checked against include/accel_dropin.h by
# tests/test_cpu_dropin.py)
$CC -w -I "$HERE/refshim" -I "$REF/include" -o "$OBJ/layout_probe" "$HERE/layout_probe.c"
"$OBJ/layout_probe" > "$OUT/accel_layout.txt"
echo "wrote $OUT/accel_layout.txt (the reference's accel.h structure layout)"
# subband dedispersion (src/dispersion.c: delay_from_dm, dedisp_delays,
# subband_delays, subband_search_delays, dedisp_subbands, float_dedisp; doppler
# from src/barycenter.c) for the dedispersion checks
$CC -O2 -g -fPIC -ffunction-sections -fdata-sections -w -I "$HERE/refshim" -I "$REF/include" \
    -c "$REF/src/dispersion.c" -o "$OBJ/dispersion.o"
$CC -O2 -g -fPIC -ffunction-sections -fdata-sections -w -I "$HERE/refshim" -I "$REF/include" \
    -c "$REF/src/barycenter.c" -o "$OBJ/barycenter.o"
echo 'REF { global: delay_from_dm; dedisp_delays; subband_delays; subband_search_delays;
      dedisp_subbands; float_dedisp; vect_free; local: *; };' > "$OUT/dedisp.map"
$CC -shared -Wl,--gc-sections -Wl,--version-script="$OUT/dedisp.map" -Wl,-z,defs \
    -o "$OUT/libref_dedisp.so" "$OBJ/dispersion.o" "$OBJ/barycenter.o" $LOBJ $SOBJ \
    "$OBJ/orc_stats.o" -fopenmp -lm
echo "built $OUT/libref_dedisp.so (src/dispersion.c)"
