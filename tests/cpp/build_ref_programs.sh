#!/bin/sh
# Compiles the reference's own OpenFHE-free test programs, unchanged and where
# they lie, against this library's headers (include/) and libgpufhe_b200.so:
# the drop-in check that a caller of the reference relinks without source
# changes. Outputs go to tests/cpp/_build/ref_programs/ (git-ignored).
#   test_rot_resident  resident rotation == host-orchestrated rotation
#   test_keyreuse      one full-QP key reused at every level
#   test_chain         15-step EvalMult / rotation / rescale chain
#   test_stage_acc     fused plaintext-multiply-accumulate
#   test_boot          the composed CKKS bootstrap
# Usage: sh tests/cpp/build_ref_programs.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT: argument, else $GPUFHE_REFERENCE_ROOT, else the recipe
#   default below. A missing tree keeps the prebuilt programs.
set -e
REF=${1:-${GPUFHE_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
OUT="$HERE/_build/ref_programs"
LIBDIR="$ROOT/gpu-resident-library_b200/gpufhe_b200"
if [ ! -d "$REF/tests" ]; then
    echo "build_ref_programs.sh: reference tree not found at $REF; keeping prebuilt $OUT" >&2
    exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
for p in test_rot_resident test_keyreuse test_chain test_stage_acc test_boot; do
    if [ ! -f "$OUT/$p" ] || [ "$REF/tests/$p.cpp" -nt "$OUT/$p" ] || [ "$LIBDIR/libgpufhe_b200.so" -nt "$OUT/$p" ] ||
       [ -n "$(find "$ROOT/include" -newer "$OUT/$p" -name '*.h')" ]; then
        "$NVCC" -std=c++17 -O2 -ccbin /usr/bin/g++ -Wno-deprecated-gpu-targets -I"$ROOT/include" \
            "$REF/tests/$p.cpp" -o "$OUT/$p" -L"$LIBDIR" -lgpufhe_b200 \
            -Xlinker -rpath -Xlinker '$ORIGIN/../../../../gpu-resident-library_b200/gpufhe_b200'
    fi
done
echo "built the reference's test programs against libgpufhe_b200.so in $OUT"
