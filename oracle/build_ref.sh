#!/bin/sh
# TEST INFRASTRUCTURE ONLY (oracle).
# Compiles the reference's own OpenCL C kernels (pyqrackising/kernels.cl, read
# in place under the reference checkout) as C with the shim in ref_shim.h, and
# links them with the ND-range emulator in ref_launch.c into
# oracle/_ref/libpqi_ref.so. The output stays out of version control.
# Usage: oracle/build_ref.sh [reference_root]
#   (default: $PQI_REFERENCE_ROOT, else the build container's /root/reference)
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${PQI_REFERENCE_ROOT:-/root/reference}}
SRC="$REF/pyqrackising/kernels.cl"
if [ ! -f "$SRC" ]; then
  echo "reference kernels not found at $SRC" >&2
  exit 1
fi
mkdir -p "$HERE/_ref"
# -ffp-contract=off keeps float sums as separate multiply/add roundings, like an
# OpenCL compile without -cl-mad-enable; -fwrapv gives the 32-bit int shift
# 1 << 31 its two's-complement value.
CFLAGS="-O2 -fPIC -std=gnu11 -fgnu89-inline -ffp-contract=off -fwrapv -w"
gcc $CFLAGS -include "$HERE/ref_shim.h" -x c -c "$SRC" -o "$HERE/_ref/kernels_ref.o"
gcc $CFLAGS -I"$HERE" -c "$HERE/ref_launch.c" -o "$HERE/_ref/ref_launch.o"
gcc -shared -o "$HERE/_ref/libpqi_ref.so" "$HERE/_ref/kernels_ref.o" "$HERE/_ref/ref_launch.o" -lpthread -lm
echo "built $HERE/_ref/libpqi_ref.so"
