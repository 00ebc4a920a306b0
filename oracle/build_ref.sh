#!/bin/bash
# Builds the reference's own SSFM code (headers included in place from the
# reference checkout) into oracle/_ref/libref_<crystal>_<size>.so.
# Test infrastructure only.  Usage: oracle/build_ref.sh [reference_root]
# The checkout is the argument, else $CUOPO_REFERENCE_ROOT, else the path
# where this build environment mounts it; this recipe is the one place that
# names it.  Without the sources (e.g. on a GPU box) it builds nothing.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUOPO_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
if [ ! -f "$REF/src/headers/cwes2.cuh" ]; then
    echo "reference sources not found under $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
# (crystal, size) variants used by the tests and the benchmark's reference arm
VARIANTS="PPLN:256 PPLN:1024 PPLN:4096 PPLN:8192 PPLN:16384 PPLN:32768 SPPLT:256 SPPLT:1024 SPPLT:65536 SPPLT:131072"
pids=()
for v in $VARIANTS; do
    cr="${v%%:*}"; sz="${v##*:}"
    lib="$OUT/libref_$(echo "$cr" | tr 'A-Z' 'a-z')_${sz}.so"
    if [ "$lib" -nt "$HERE/ref_harness.cu" ] && [ "$lib" -nt "$HERE/build_ref.sh" ]; then continue; fi
    "$NVCC" "$HERE/ref_harness.cu" -I"$REF/src" -D"$cr" -DREF_SIZE="$sz" \
        -diag-suppress 177,550 -gencode arch=compute_100a,code=sm_100a \
        -Xcompiler -fPIC -shared -lcufft -o "$lib" &
    pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
exit $rc
