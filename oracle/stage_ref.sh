#!/bin/sh
# Oracle test infrastructure: stage a patched copy of the reference sources
# into the git-ignored build folder. Usage: stage_ref.sh <reference root> <out>
set -e
REF="$1"; OUT="$2"
test -d "$REF/src" || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
rm -rf "$OUT/src" "$OUT/bin" "$OUT/dependencies"
cp -r "$REF/src" "$OUT/src"
cp -r "$REF/bin" "$OUT/bin"
mkdir -p "$OUT/dependencies/include"
cp -r "$REF/dependencies/include/glm" "$OUT/dependencies/include/glm"
cp -r "$REF/dependencies/include/cgltf" "$OUT/dependencies/include/cgltf"
cp -r "$REF/dependencies/include/stb" "$OUT/dependencies/include/stb"
chmod -R u+w "$OUT"
# src/core/util.h:60-105 — `-> typename enable_if_t<...>` is accepted only by MSVC.
sed -i 's/-> typename enable_if_t</-> enable_if_t</' "$OUT/src/core/util.h"
# src/core/util.h:28 — host code sees CUdeviceptr; the CPU launch needs real pointers.
sed -i 's/#    define CUPTR(type) CUdeviceptr/#    define CUPTR(type) type*/' "$OUT/src/core/util.h"
