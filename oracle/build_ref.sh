#!/bin/sh
# Rebuilds the reference library from its own sources, where they lie, into
# oracle/_ref/ (git-ignored) for parity pins. Nothing is copied out of the
# reference tree; its sources are compiled in place, read-only.
#   libref_host.so : params.cpp + ks_constants.cpp + encode.cpp (CPU only)
#   libref_gpu.so  : every src/*.cpp and kernels/*.cu for sm_100a
#   ref_test_boot  : the reference's composed-bootstrap test program
#                    (tests/test_boot.cpp) with the same sources, for timing
#                    the reference's own bootstrap beside this library's
# Usage: sh oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -e
REF=${1:-${REF:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    echo "build_ref.sh: reference tree not found at $REF; keeping prebuilt $OUT" >&2
    exit 0
fi
mkdir -p "$OUT"
/usr/bin/g++ -O2 -std=gnu++17 -fPIC -shared -I"$REF/include" \
    "$REF/src/params.cpp" "$REF/src/ks_constants.cpp" "$REF/src/encode.cpp" \
    "$HERE/ref_shim_host.cpp" -o "$OUT/libref_host.so"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
"$NVCC" -std=c++17 -O2 -Xcompiler -fPIC -shared -ccbin /usr/bin/g++ \
    -gencode arch=compute_100a,code=sm_100a \
    -I"$REF/include" "$REF"/src/*.cpp "$REF"/kernels/*.cu \
    "$HERE/ref_shim_gpu.cpp" -Xlinker -Bsymbolic -o "$OUT/libref_gpu.so"
"$NVCC" -std=c++17 -O2 -ccbin /usr/bin/g++ -gencode arch=compute_100a,code=sm_100a \
    -I"$REF/include" "$REF"/src/*.cpp "$REF"/kernels/*.cu "$REF/tests/test_boot.cpp" \
    -o "$OUT/ref_test_boot"
echo "built $OUT/libref_host.so $OUT/libref_gpu.so $OUT/ref_test_boot"
