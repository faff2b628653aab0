#!/bin/sh
# ORACLE — test infrastructure only.  Compiles the reference's sap/graph.h
# (from the reference source tree given as $1, default /root/reference)
# against the CUSP stand-in in this directory into oracle/_ref/libref_graph.so.
# Nothing from the reference tree is copied; the output stays out of git.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-/root/reference}
OUT="$HERE/../_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
[ -f "$REF/sap/graph.h" ] || { echo "reference tree not found at $REF" >&2; exit 2; }
mkdir -p "$OUT"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -Xcompiler -fPIC -shared \
    -w -I "$HERE" -I "$REF" "$HERE/ref_graph_driver.cu" -o "$OUT/libref_graph.so"
echo "$OUT/libref_graph.so"
