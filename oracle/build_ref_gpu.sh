#!/bin/bash
# TEST INFRASTRUCTURE ONLY.
# Builds the reference's own GPU kernels (minimum_lbvh.cu and main_gpu.cu, compiled from the
# sources where they lie, for sm_100a) with the host launchers in oracle/ref_gpu_lbvh.cu and
# oracle/ref_gpu_main.cu into two git-ignored libraries that travel with the working tree to
# the GPU box (where the reference sources are absent):
#   oracle/_ref/libpzref_gpu.so        the compiler's default FMA contraction, as the
#                                      reference's run-time compile builds them (timing);
#   oracle/_ref/libpzref_gpu_exact.so  -fmad=false: the reference's CPU float arithmetic (parity).
# No reference source is copied into the repository.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference sources: $REF_DIR, else a directory named "reference" beside the repository
REF_DIR=${REF_DIR:-$(cd "$HERE/../.." && pwd)/reference}
OUT=$HERE/_ref
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -f "$REF_DIR/main_gpu.cu" ] || [ ! -f "$REF_DIR/minimum_lbvh.cu" ]; then
  echo "build_ref_gpu.sh: reference sources not found at $REF_DIR; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/gpu"
ARCH="-gencode arch=compute_100a,code=sm_100a"
COMMON="-O3 -std=c++17 -Xcompiler -fPIC -w -I$REF_DIR"
for variant in default exact; do
  FLAGS=""
  SUFFIX=""
  if [ "$variant" = exact ]; then FLAGS="-fmad=false"; SUFFIX="_exact"; fi
  # ref_gpu_main.cu includes ref_gpu_lbvh.cu: one translation unit
  $NVCC $ARCH $COMMON $FLAGS -I"$HERE" -c "$HERE/ref_gpu_main.cu" -o "$OUT/gpu/main$SUFFIX.o"
  $NVCC $ARCH -shared -o "$OUT/libpzref_gpu$SUFFIX.so" "$OUT/gpu/main$SUFFIX.o"
done
echo "built $OUT/libpzref_gpu.so $OUT/libpzref_gpu_exact.so"
