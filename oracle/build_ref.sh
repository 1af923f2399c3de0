#!/bin/sh
# Compiles the reference's own OpenCL block-matching kernel
# (src/mirorr/kernels/optKmatchMask.cl) for the CPU, through the OpenCL-C
# emulation in oracle/ref_shim/optkmatch_cpu.cpp.  Reads the kernel source in
# place from the reference tree; writes only oracle/_ref/liboptkmatch_ref.so.
# Test infrastructure: the result pins the oracle's NCC search.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${MIRORR_REFERENCE:-/root/reference}
CL="$REF/src/mirorr/kernels/optKmatchMask.cl"
if [ ! -f "$CL" ]; then
  echo "reference kernel not found at $CL" >&2
  exit 2
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -ffp-contract=off -fno-fast-math -fPIC -shared -pthread \
    -DOPTKMATCH_CL="\"$CL\"" \
    "$HERE/ref_shim/optkmatch_cpu.cpp" -o "$HERE/_ref/liboptkmatch_ref.so.tmp"
mv "$HERE/_ref/liboptkmatch_ref.so.tmp" "$HERE/_ref/liboptkmatch_ref.so"
echo "$HERE/_ref/liboptkmatch_ref.so"
