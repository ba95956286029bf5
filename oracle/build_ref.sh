#!/usr/bin/env bash
# Test infrastructure: compile the reference's vendored FastQSL adaptive
# tracer (TraceBlineAdaptive.cu, from where it lies in the reference tree)
# with the launcher oracle/fastqsl_ref_launch.cu into oracle/_ref/.  The
# library is used only by tests/golden/make_fastqsl_golden.py to write
# fixtures; the product never loads it.
set -euo pipefail
REF="${NFGS_REFERENCE:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
SRC="$REF/third_party/FastQSL/fastqslpy/cu"
NVCC="${NVCC:-$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)}"
if [ ! -f "$SRC/TraceBlineAdaptive.cu" ]; then
    echo "reference sources absent: oracle/_ref not rebuilt"
    exit 0
fi
mkdir -p "$HERE/_ref"
"$NVCC" -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared \
    -diag-suppress 177,550,1444,2464 -Xcompiler -w -I "$SRC" "$HERE/fastqsl_ref_launch.cu" -o "$HERE/_ref/libfastqsl_ref.so"
echo "built $HERE/_ref/libfastqsl_ref.so"
