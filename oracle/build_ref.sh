#!/bin/sh
# Rebuilds the reference library from its own sources, where they lie, into
# oracle/_ref/ (git-ignored) for parity pins. Nothing is copied out of the
# reference tree; its sources are compiled in place, read-only.
#   libref_host.so : params.cpp + ks_constants.cpp + encode.cpp (CPU only)
#   libref_gpu.so  : every src/*.cpp and kernels/*.cu for sm_100a
#   ref_<program>  : the reference's OpenFHE-free test programs
#                    (tests/test_boot.cpp, test_rot_resident.cpp,
#                    test_keyreuse.cpp, test_chain.cpp, test_stage_acc.cpp)
#                    linked with the reference's own sources, so their output
#                    and timing sit beside the same programs linked against
#                    this library (tests/cpp/build_ref_programs.sh)
# Usage: sh oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT: argument, else $GPUFHE_REFERENCE_ROOT, else the recipe
#   default below. A missing tree keeps the prebuilt outputs.
set -e
REF=${1:-${GPUFHE_REFERENCE_ROOT:-/root/reference}}
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
# the library's objects once, then one link per test program
OBJ="$OUT/obj"
mkdir -p "$OBJ"
for f in "$REF"/src/*.cpp "$REF"/kernels/*.cu; do
    b=$(basename "$f")
    if [ ! -f "$OBJ/$b.o" ] || [ "$f" -nt "$OBJ/$b.o" ]; then
        "$NVCC" -std=c++17 -O2 -ccbin /usr/bin/g++ -gencode arch=compute_100a,code=sm_100a \
            -I"$REF/include" -c "$f" -o "$OBJ/$b.o"
    fi
done
for p in test_boot test_rot_resident test_keyreuse test_chain test_stage_acc; do
    "$NVCC" -std=c++17 -O2 -ccbin /usr/bin/g++ -gencode arch=compute_100a,code=sm_100a \
        -I"$REF/include" "$REF/tests/$p.cpp" "$OBJ"/*.o -o "$OUT/ref_$p"
done
echo "built $OUT/libref_host.so $OUT/libref_gpu.so and the reference's test programs in $OUT"
