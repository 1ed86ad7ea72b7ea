#!/bin/sh
# Compiles the parts of the reference's accelsearch path that build from the
# reference's own source files with no external library, into oracle/_ref/.
# Only src/fresnl.c (Cephes Fresnel integrals, used by gen_z_response at
# src/responses.c:291-292) qualifies: every other hot-path file includes
# ransomfft.h -> fftw3.h, or needs GSL / glib, none of which exist here.
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
