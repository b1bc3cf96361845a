#!/usr/bin/env bash
# Builds the reference solver from its own sources, in place under the
# read-only reference tree, into oracle/_ref/ (git-ignored test infrastructure):
#   libref_<v>_gpu.so : full reference step (nvcc, sm_100a) + ref_driver.cpp
#   libref_<v>_mc.so  : reference CPU marching cubes (host only) + ref_mc_driver.cpp
# v in {2d, 3d2, 3d4}; the _mc library exists for the 3D variants only.
# The only project-written code compiled in is oracle/ref_shim/cutil_math.h
# (stand-in for the retired SDK header) and the two drivers.
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or SCA2012_REFERENCE=REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${SCA2012_REFERENCE:-}}"
if [ -z "$REF" ]; then
  echo "build_ref: no reference root given (argument or SCA2012_REFERENCE); keeping existing oracle/_ref" >&2
  exit 0
fi
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF/SPH-3D-2" ]; then
  echo "build_ref: reference tree not found at $REF; keeping existing $OUT" >&2
  exit 0
fi
NVCC="${NVCC:-nvcc}"
ARCH="-gencode arch=compute_100a,code=sm_100a"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT

build_variant() {
  local v="$1" dir="$2" dim="$3"
  local src="$REF/$dir"
  # The reference .cu includes "sph_kernel.cu" and the headers by relative
  # name, so compile from the reference directory with -I for the shim.
  # Objects go to a temp dir; nothing is written into the reference tree.
  "$NVCC" $ARCH -O2 -std=c++14 -Xcompiler -fPIC -I"$HERE/ref_shim" -I"$src" \
      -x cu -c "$src/sph_system.cu" -o "$TMP/${v}_sys_cu.o" -w
  "$NVCC" $ARCH -O2 -std=c++14 -Xcompiler -fPIC -I"$HERE/ref_shim" -I"$src" \
      -x cu -c "$src/sph_system.cpp" -o "$TMP/${v}_sys_cpp.o" -w
  "$NVCC" $ARCH -O2 -std=c++14 -Xcompiler -fPIC -I"$HERE/ref_shim" -I"$src" \
      -DREF_DIM=$dim -x cu -c "$HERE/ref_driver.cpp" -o "$TMP/${v}_drv.o" -w
  "$NVCC" $ARCH -shared "$TMP/${v}_sys_cu.o" "$TMP/${v}_sys_cpp.o" "$TMP/${v}_drv.o" \
      -o "$OUT/libref_${v}_gpu.so"
  if [ "$dim" = 3 ]; then
    "$NVCC" -O2 -std=c++14 -Xcompiler -fPIC -I"$HERE/ref_shim" -I"$src" \
        -x cu -c "$src/sph_system.cpp" -o "$TMP/${v}_mc_sys.o" -w $ARCH
    "$NVCC" -O2 -std=c++14 -Xcompiler -fPIC -I"$HERE/ref_shim" -I"$src" \
        -x cu -c "$HERE/ref_mc_driver.cpp" -o "$TMP/${v}_mc_drv.o" -w $ARCH
    "$NVCC" $ARCH -shared "$TMP/${v}_mc_sys.o" "$TMP/${v}_mc_drv.o" -o "$OUT/libref_${v}_mc.so"
  fi
}

build_variant 2d SPH-2D 2
build_variant 3d2 SPH-3D-2 3
build_variant 3d4 SPH-3D-4 3
echo "build_ref: built $(ls "$OUT" | tr '\n' ' ')"
