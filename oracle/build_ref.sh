#!/usr/bin/env bash
# Build oracle/_ref/libref_rrtm.so: the reference's own RRTM kernel sources (read in place from the
# reference tree, never copied) compiled as host C++ behind oracle/ref_shim.h and driven by
# oracle/ref_driver.cpp.  Needs the reference tree, given as the first argument or as WOOF_NAM_REFERENCE;
# machines without it use the prebuilt library.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${WOOF_NAM_REFERENCE:-}}"
if [ -z "$REF" ]; then
    echo "usage: build_ref.sh <reference tree>   (or set WOOF_NAM_REFERENCE)" >&2
    exit 2
fi
KDIR="$REF/namgpu/kernels"
if [ ! -d "$KDIR" ]; then
    echo "build_ref.sh: reference kernels not found at $KDIR" >&2
    exit 1
fi
mkdir -p "$HERE/_ref"
g++ -std=c++17 -O2 -ffp-contract=off -fopenmp -fPIC -shared -w \
    -I "$KDIR" -o "$HERE/_ref/libref_rrtm.so" "$HERE/ref_driver.cpp"
echo "built $HERE/_ref/libref_rrtm.so"
