#!/usr/bin/env bash
# Builds oracle/_ref/libhp_ref.so: the reference's own CPU contraction, edge
# cut, graph split and CPU coarsening, compiled from the reference sources in place
# (REF_DIR, default /root/reference) through oracle/ref_harness.cu.
# TEST INFRASTRUCTURE ONLY; output stays in oracle/_ref/ (git-ignored).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/HunyuanGRAPH.h" ]; then
  echo "reference sources not found at $REF_DIR; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
nvcc -std=c++14 -O2 -w --expt-relaxed-constexpr \
  -gencode arch=compute_100a,code=sm_100a \
  -Xcompiler -fPIC -shared -I "$REF_DIR" \
  -o "$OUT/libhp_ref.so" "$HERE/ref_harness.cu"
echo "$OUT/libhp_ref.so"
