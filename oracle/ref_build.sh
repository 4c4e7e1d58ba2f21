#!/bin/bash
# Builds the reference project's own preprocessing CLI (host C++ only) from its
# sources where they lie, into oracle/_ref/.  Test infrastructure: the CPU
# tests run it to pin the tokenizer's token and term counts.  The reference's
# join is CUDA and is not built or run here.
set -e
REF=${FGSS_REFERENCE:-/root/reference}  # where the reference checkout lies
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -d "$REF/src" ] || { echo "reference sources not found at $REF; nothing to build"; exit 0; }
mkdir -p "$OUT"
g++ -O2 -std=c++11 -w \
    -I"$REF/include" -I"$REF/include/preprocess/string" \
    "$REF/src/preprocess_cli.cpp" "$REF/src/preprocess/string/preprocess.cpp" \
    "$REF/src/preprocess/string/data.cpp" "$REF/src/preprocess/string/qgram.cpp" \
    "$REF/src/io.cpp" "$REF/src/util.cpp" -o "$OUT/preprocess"
echo "built $OUT/preprocess"
