#!/usr/bin/env bash
# Builds oracle/_ref/libcvrp_ref.so: the reference's own host code
# (cvrp_ocl/{problem,io,vrpHelper,utilities,unix_timer,localSearch,neighbourSearch,move}.cpp, gpu/g_type.cpp,
# gpu/g_aco.cpp) and its OpenCL kernels (gpu/kernel.cl, compiled as C++) linked
# against the fake OpenCL runtime in oracle/refshim.  Test infrastructure only.
#
# Usage: oracle/build_ref.sh [REFERENCE_DIR]   (default $CVRP_REFERENCE_DIR, else /root/reference)
# Intermediate files go to a temporary directory; only the .so lands in oracle/_ref/.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${1:-${CVRP_REFERENCE_DIR:-/root/reference}}"
SRC="$REF_ROOT/cvrp_ocl"
OUT="$HERE/_ref"
if [ ! -f "$SRC/gpu/kernel.cl" ]; then
  echo "build_ref: reference sources not found under $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT

CXX="${CXX:-g++}"
FLAGS=(-O2 -std=gnu++11 -ffp-contract=off -fPIC -w)
INC=(-I"$HERE/refshim" -I"$SRC" -I"$SRC/gpu")

# kernel.cl as C++: __local variables declared inside a kernel body become
# function statics (shared by the emulated work-group); everything else is
# handled by the kernel_shim.h macros.  The kernels live in namespace oclk.
{
  echo '#include "kernel_shim.h"'
  echo 'namespace oclk {'
  echo '#line 1 "kernel.cl"'
  sed -E 's/^([[:space:]]+)__local([[:space:]]+[A-Za-z_]+[[:space:]]+[A-Za-z_]+;)/\1static\2/' "$SRC/gpu/kernel.cl"
  echo '}'
} > "$TMP/kernel_cl.cpp"

objs=()
for f in problem io vrpHelper utilities unix_timer localSearch neighbourSearch move; do
  "$CXX" "${FLAGS[@]}" "${INC[@]}" -c "$SRC/$f.cpp" -o "$TMP/$f.o"
  objs+=("$TMP/$f.o")
done
for f in g_type g_aco; do
  "$CXX" "${FLAGS[@]}" "${INC[@]}" -c "$SRC/gpu/$f.cpp" -o "$TMP/$f.o"
  objs+=("$TMP/$f.o")
done
"$CXX" "${FLAGS[@]}" -I"$HERE/refshim" -c "$TMP/kernel_cl.cpp" -o "$TMP/kernel_cl.o"
"$CXX" "${FLAGS[@]}" "${INC[@]}" -c "$HERE/refshim/fakecl.cpp" -o "$TMP/fakecl.o"
"$CXX" "${FLAGS[@]}" "${INC[@]}" -c "$HERE/refshim/ref_driver.cpp" -o "$TMP/ref_driver.o"
"$CXX" -shared -Wl,-Bsymbolic -Wl,--exclude-libs,ALL -o "$OUT/libcvrp_ref.so" "${objs[@]}" \
  "$TMP/kernel_cl.o" "$TMP/fakecl.o" "$TMP/ref_driver.o" -lm
echo "build_ref: wrote $OUT/libcvrp_ref.so"
