#!/usr/bin/env bash
# Test infrastructure: builds the reference Tractor's own C kernels into
# oracle/_ref/ so that the oracle can be checked against them.
#
# The reference compiles these with SWIG (tractor/mix.i, tractor/mp_fourier.i,
# tractor/emfit.i);
# SWIG is not installed here, so this recipe copies the C text of the
# `%{ ... %}` and `%inline %{ ... %}` blocks out of the .i files (by block
# markers, verbatim) into oracle/_ref/, and compiles it together with a small
# shim (oracle/ref_shim_mix.c, oracle/ref_shim_mpf.c, oracle/ref_shim_emfit.c)
# that only adds exported entry points.  approx3.c, gauss_masked.c and
# emfit2.c are #included from where they lie in the reference tree.  Nothing here is used by the product path.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
# The tree is the argument, else $TRACTOR_REFERENCE_ROOT, else the build
# container's read-only copy; when none holds tractor/mix.i nothing is built
# (the GPU machines have no reference tree and use the files built here).
# The tree used is recorded in oracle/_ref/REFERENCE_ROOT for the Python
# harness (oracle/refharness.py) and the tests that read reference files.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${TRACTOR_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -f "$REF/tractor/mix.i" ]; then
    echo "build_ref.sh: reference tree not found at $REF; nothing built" >&2
    exit 0
fi
mkdir -p "$OUT"
printf '%s\n' "$REF" > "$OUT/REFERENCE_ROOT"

# Print the bodies of every %{ ... %} / %inline %{ ... %} block, skipping %init.
extract() {
    awk '
        /^%init[ \t]*%\{/            { skip = 1; next }
        /^%\{/ || /^%inline[ \t]*%\{/ { inblk = 1; next }
        /^[ \t]*%\}/                 { inblk = 0; skip = 0; next }
        inblk && !skip               { print }
    ' "$1"
}
extract "$REF/tractor/mix.i"        > "$OUT/ref_mix_blocks.c"
extract "$REF/tractor/mp_fourier.i" > "$OUT/ref_mpf_blocks.c"
extract "$REF/tractor/emfit.i"      > "$OUT/ref_emfit_blocks.c"

PYINC="$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["include"])')"
NPINC="$(python3 -c 'import numpy; print(numpy.get_include())')"
CFLAGS="-O2 -fPIC -shared -std=gnu99 -w"

gcc $CFLAGS -I"$OUT" -I"$REF/tractor" -I"$PYINC" -I"$NPINC" \
    "$HERE/ref_shim_mix.c" -o "$OUT/libref_mix.so" -lm
gcc $CFLAGS -I"$OUT" -I"$REF/tractor" -I"$PYINC" -I"$NPINC" \
    "$HERE/ref_shim_mpf.c" -o "$OUT/libref_mpf.so" -lm
gcc $CFLAGS -I"$OUT" -I"$REF/tractor" -I"$PYINC" -I"$NPINC" \
    "$HERE/ref_shim_emfit.c" -o "$OUT/libref_emfit.so" -lm
echo "built $OUT/libref_mix.so $OUT/libref_mpf.so $OUT/libref_emfit.so"
