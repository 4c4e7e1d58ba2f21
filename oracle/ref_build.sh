#!/bin/bash
# Builds, into oracle/_ref/, test infrastructure from the reference project's
# own sources where they lie (nothing is copied): the CPU tests run these to pin
# the oracle and the library against the reference's code.
#   preprocess   its preprocessing CLI (host C++): token and term counts
#   ref_bounds   oracle/ref_bounds.cpp over its include/fgssjoin/similarity.cuh,
#                compiled on the host: the float32 bound tables
#   ref_load     oracle/ref_load.cu over its src/fgssjoin/data.cu loader
#                (ppjoin_format, host code only): the .bin record order
#   ref_join     oracle/ref_join.cu over its join kernels (data, index,
#                filtering, checking, compaction, util): the reference's own
#                GPU join with one tile, run by the GPU tests on a B200
set -e
REF=${FGSS_REFERENCE:-/root/reference}  # where the reference checkout lies
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
[ -d "$REF/src" ] || { echo "reference sources not found at $REF; nothing to build"; exit 0; }
mkdir -p "$OUT"
g++ -O2 -std=c++11 -w \
    -I"$REF/include" -I"$REF/include/preprocess/string" \
    "$REF/src/preprocess_cli.cpp" "$REF/src/preprocess/string/preprocess.cpp" \
    "$REF/src/preprocess/string/data.cpp" "$REF/src/preprocess/string/qgram.cpp" \
    "$REF/src/io.cpp" "$REF/src/util.cpp" -o "$OUT/preprocess"
echo "built $OUT/preprocess"
# strict IEEE float, no FMA contraction: the expressions round as written
g++ -O2 -std=c++11 -w -fno-fast-math -ffp-contract=off -I"$REF/include/fgssjoin" \
    "$HERE/ref_bounds.cpp" -o "$OUT/ref_bounds"
echo "built $OUT/ref_bounds"
if [ "$HERE/ref_load.cu" -nt "$OUT/ref_load" ] || [ ! -x "$OUT/ref_load" ]; then
    "$NVCC" -O2 -std=c++14 -w -gencode arch=compute_100a,code=sm_100a \
        -I"$REF/include" -I"$REF/include/fgssjoin" \
        "$HERE/ref_load.cu" "$REF/src/fgssjoin/data.cu" "$REF/src/util.cu" "$REF/src/util.cpp" "$REF/src/io.cpp" \
        -o "$OUT/ref_load" -lcuda
    echo "built $OUT/ref_load"
fi
if [ "$HERE/ref_join.cu" -nt "$OUT/ref_join" ] || [ ! -x "$OUT/ref_join" ]; then
    "$NVCC" -O3 -std=c++14 -w -gencode arch=compute_100a,code=sm_100a \
        -I"$REF/include" -I"$REF/include/fgssjoin" \
        "$HERE/ref_join.cu" "$REF/src/fgssjoin/data.cu" "$REF/src/fgssjoin/index.cu" \
        "$REF/src/fgssjoin/filtering.cu" "$REF/src/fgssjoin/checking.cu" "$REF/src/fgssjoin/compaction.cu" \
        "$REF/src/util.cu" "$REF/src/util.cpp" "$REF/src/io.cpp" -o "$OUT/ref_join"
    echo "built $OUT/ref_join"
fi
