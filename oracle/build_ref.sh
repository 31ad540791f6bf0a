#!/usr/bin/env bash
# Compiles the reference's GPU BCD solver from its own sources, read in place
# under <reference checkout>/src, plus oracle/ref_bcd_shim.cu, into
# oracle/_ref/libref_bcd.so (git-ignored; travels to the GPU box with the
# repository snapshot).  Only the BCD path builds here: the reference's SPLR
# sources need cuDSS and CCCL >= 3.1, neither of which is in this image.
#
# Usage: build_ref.sh <reference checkout>   (or set REFERENCE_ROOT)
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
root="${1:-${REFERENCE_ROOT:-}}"
out="$here/_ref"
if [ -z "$root" ]; then
  echo "no reference checkout given; keeping prebuilt $out" >&2
  exit 0
fi
src="$root/src"
if [ ! -f "$src/sinkhorn_bcd_kernel.cu" ]; then
  echo "reference sources not found at $src; keeping prebuilt $out" >&2
  exit 0
fi
mkdir -p "$out"
arch="-gencode arch=compute_100a,code=sm_100a"
nvcc $arch -O2 -std=c++17 -Xcompiler -fPIC -I"$src" -shared \
  "$src/sinkhorn_bcd_kernel.cu" "$src/utils.cu" "$here/ref_bcd_shim.cu" \
  -o "$out/libref_bcd.so"
echo "built $out/libref_bcd.so"
