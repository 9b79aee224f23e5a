#!/usr/bin/env bash
# Builds baseline/_ref/hunyuangraph_sm100a: the reference's own GPU partitioner
# (its command-line program hunyuangraph.cu with every header it includes) for
# sm_100a.  The sources are copied to a temporary directory because SM_NUM must
# be set to this GPU's SM count (148 on a B200) as the reference's own make.sh
# does with sed (make.sh:46-63); nothing else is changed.  The flags are the
# reference Makefile's (-O3 --expt-relaxed-constexpr -w) with the target arch.
# Output stays in baseline/_ref/ (git-ignored; it travels with the snapshot).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
SM="${SM_NUM:-148}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/hunyuangraph.cu" ]; then
  echo "reference sources not found at $REF_DIR; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
cp "$REF_DIR"/*.h "$REF_DIR"/hunyuangraph.cu "$TMP"/
sed -i "s/^#define SM_NUM .*/#define SM_NUM $SM/" "$TMP/hunyuangraph_define.h"
nvcc -std=c++11 -gencode arch=compute_100a,code=sm_100a -O3 --expt-relaxed-constexpr -w \
  -o "$OUT/hunyuangraph_sm100a" "$TMP/hunyuangraph.cu"
echo "$OUT/hunyuangraph_sm100a"
