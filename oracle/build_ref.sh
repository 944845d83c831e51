#!/usr/bin/env bash
# build_ref.sh -- TEST INFRASTRUCTURE ONLY.
# Compiles the reference implementation from its own sources, where they lie,
# into oracle/_ref/ (git-ignored; travels with the repository snapshot):
#   oracle/_ref/libperman_ref.so  -- reference functions behind extern "C" shims
#   oracle/_ref/perman_ref        -- the reference CLI, unmodified
# The reference's own Makefile is not used.  Flags follow its build line
# (Makefile:2) plus -include cstdint (util.h uses INT8_MAX without <cstdint>)
# and an sm_100a target.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# $REF_SRC, else a `reference` directory beside this repository
REF=${REF_SRC:-$HERE/../../reference}
OUT="$HERE/_ref"
if [ ! -f "$REF/main.cu" ]; then
  echo "reference sources not found at $REF; keeping prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
$NVCC -O3 $ARCH -std=c++14 -Xcompiler -fopenmp -Xcompiler -fPIC -include cstdint \
  -I"$REF" -shared -o "$OUT/libperman_ref.so" "$HERE/ref_harness.cu" -lgomp -w
$NVCC -O3 $ARCH -Xcompiler -fopenmp -include cstdint -o "$OUT/perman_ref" "$REF/main.cu" -lgomp -w
echo "built $OUT/libperman_ref.so and $OUT/perman_ref"
