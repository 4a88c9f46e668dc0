#!/bin/bash
# TEST INFRASTRUCTURE ONLY.
# Builds the reference's own CPU code, from the sources where they lie, into
# oracle/_ref/libpzref.so (git-ignored; it travels with the working tree to the
# GPU box, where the reference sources are absent).  The shims in
# oracle/ref_shims stand in for the Windows, PPL and Orochi headers; pk_oracle.h is
# generated from pk.h by dropping line 4 (the GPU-builder define) and the renderer
# class (lines 1171-1704 plus the matching #endif on line 2224), which needs the
# absent graphics/Alembic libraries.  No reference source is copied into the repo.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference sources: $REF_DIR, else a directory named "reference" beside the repository
REF_DIR=${REF_DIR:-$(cd "$HERE/../.." && pwd)/reference}
OUT=$HERE/_ref
if [ ! -f "$REF_DIR/pk.h" ]; then
  echo "build_ref.sh: reference sources not found at $REF_DIR; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/gen"
# guard the line-based excision against a different pk.h
sed -n '4p' "$REF_DIR/pk.h" | grep -q '^#define ENABLE_GPU_BUILDER' || { echo "unexpected pk.h line 4" >&2; exit 1; }
sed -n '1171p' "$REF_DIR/pk.h" | grep -q '^#if !defined(PK_KERNELCC)' || { echo "unexpected pk.h line 1171" >&2; exit 1; }
sed -n '1705p' "$REF_DIR/pk.h" | grep -q '^struct InternalNormalBound' || { echo "unexpected pk.h line 1705" >&2; exit 1; }
sed -n '2224p' "$REF_DIR/pk.h" | grep -q '^#endif' || { echo "unexpected pk.h line 2224" >&2; exit 1; }
sed -n '1,3p;5,1170p;1705,2222p' "$REF_DIR/pk.h" > "$OUT/gen/pk_oracle.h"
CXX=/usr/bin/g++
[ -x "$CXX" ] || CXX=g++
$CXX -std=c++17 -O2 -fPIC -fopenmp -ffp-contract=off -fno-fast-math -w -shared \
  -I"$HERE/ref_shims" -I"$OUT/gen" -I"$REF_DIR" \
  -include "$HERE/ref_shims/std_expf.h" -include memory -include cstdio -include cstring -include algorithm \
  -o "$OUT/libpzref.so" "$HERE/ref_harness.cpp"
echo "built $OUT/libpzref.so"
