#!/bin/bash
# Builds the reference LucasNTT program from its sources, read in place and
# never copied, into oracle/_ref/LucasNTT (sm_100, CUDA 12.9).
#
# Test infrastructure: the GPU parity tests and oracle/run_ref.py run this
# binary on a B200 to pin residues and timings against the reference's own
# build.  The reference needs `--pre-include cstdint` with this nvcc/gcc
# (common/common.cuh uses uint32_t without including <cstdint>).
#
# Usage: oracle/build_ref.sh [REFERENCE_DIR]; the directory defaults to
# $LNT_REFERENCE_DIR, else to where this build's reference checkout lives.
set -euo pipefail
REF=${1:-${LNT_REFERENCE_DIR:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF" ]; then
    echo "build_ref: no reference sources at $REF; keeping the prebuilt binary if any"
    exit 0
fi
NVCC=${NVCC:-nvcc}
GENCODE="-gencode=arch=compute_100,code=sm_100"
mkdir -p "$OUT/obj"
BIN="$OUT/LucasNTT"
if [ -x "$BIN" ] && [ -z "$(find "$REF" -type f \( -name '*.cu' -o -name '*.cpp' -o -name '*.cuh' -o -name '*.h' \) -newer "$BIN" -print -quit)" ]; then
    echo "build_ref: $BIN is up to date"
    exit 0
fi
export NVCC GENCODE OUT REF
find "$REF" -type f \( -name '*.cu' -o -name '*.cpp' \) -print0 |
    xargs -0 -P "${JOBS:-8}" -I{} bash -c '
        src="$1"; rel="${src#$REF/}"; obj="$OUT/obj/${rel//\//__}.o"
        $NVCC $GENCODE --pre-include cstdint -O2 -Xcompiler -O2 -c "$src" -o "$obj"
    ' _ {}
$NVCC $GENCODE -o "$BIN" "$OUT"/obj/*.o
echo "build_ref: built $BIN"
