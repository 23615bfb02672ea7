#!/usr/bin/env bash
# Builds the reference's own CUDA sources, unmodified, once per case, into
# oracle/_ref/ref_<case> (test infrastructure: parity fixtures and the
# reference arm of bench.py).  Needs the reference checkout; the built
# binaries travel with the repository snapshot, the sources do not.
#
# The reference is configured by compile-time constants only, so each case
# pre-includes a generated header (oracle/ref_constants.py) that defines the
# reference's CONSTANTS_CUH guard and all its constants.  Flags follow the
# reference's compile.sh (-O3 -std=c++20 --extended-lambda -rdc=true) with the
# architecture set to sm_100a.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${MCG_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/kernels.cu" ]; then
    echo "build_ref.sh: reference sources not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
# where the sources were found, for tests that read the reference's post/
# scripts in this checkout (oracle/_ref/ is a build folder, not committed)
echo "$REF" > "$OUT/REFERENCE_DIR"
PY="${PYTHON:-python}"
CASES="${MCG_REF_CASES:-$("$PY" "$HERE/ref_constants.py" --list)}"
for c in $CASES; do
    hdr="$OUT/$c/constants_case.cuh"
    "$PY" "$HERE/ref_constants.py" "$c" "$hdr"
    bin="$OUT/ref_$c"
    if [ -x "$bin" ] && [ "$bin" -nt "$hdr" ] && [ "$bin" -nt "$HERE/ref_dump.cu" ]; then
        continue
    fi
    # separate object dir per case keeps parallel builds apart
    obj="$OUT/$c"
    nvcc -O3 -std=c++20 --extended-lambda -rdc=true \
        -gencode arch=compute_100a,code=sm_100a \
        -include "$hdr" -I "$REF" \
        -c "$REF/kernels.cu" -o "$obj/kernels.o"
    nvcc -O3 -std=c++20 --extended-lambda -rdc=true \
        -gencode arch=compute_100a,code=sm_100a \
        -include "$hdr" -I "$REF" \
        -c "$HERE/ref_dump.cu" -o "$obj/ref_dump.o"
    nvcc -rdc=true -gencode arch=compute_100a,code=sm_100a \
        "$obj/kernels.o" "$obj/ref_dump.o" -o "$bin"
    echo "built $bin"
done
