#!/bin/sh
# Regenerate xsec_*.txt from the reference's own table builder
# (src/PhysicsData.c).  Development-time only: needs the reference tree.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference tree: $REF, by default the directory `reference` beside this repository
REF=${REF:-$(cd "$HERE/../../.." && pwd)/reference}
TMP=$(mktemp -d)
gcc -c -O1 -w -I"$REF/inc" "$REF/src/PhysicsData.c" -o "$TMP/PhysicsData.o"
nvcc -c -w -Wno-deprecated-gpu-targets -I"$REF/inc" "$REF/src/Variables.cu" -o "$TMP/Variables.o"
gcc -c -O1 -w -I"$REF/inc" "$HERE/gen_xsec_tables.c" -o "$TMP/gen.o"
g++ -o "$TMP/gen" "$TMP"/*.o -L/usr/local/cuda/lib64 -lcudart_static -ldl -lpthread -lrt -lm
"$TMP/gen" "$HERE"
rm -rf "$TMP"
