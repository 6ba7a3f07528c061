#!/bin/bash
# Test infrastructure only: compiles the reference solver's OWN sources, read
# in place from $REF_DIR (required: the reference checkout), together with the shims in
# oracle/shims and the driver oracle/ref_harness.cpp, into oracle/_ref/.
# Two flavours are built:
#   o2f_ref_exact  -O2 -ffp-contract=off   parity oracle (no fused multiply-add)
#   o2f_ref_fast   -O3 -march=x86-64-v3    timed CPU baseline (OpenMP)
# shape_optimization.cpp is compiled without its Eigen-based solver and
# optimizeShape (lines 560-741 and 1017-): Eigen is not installed.  The
# extract is generated under oracle/_ref/ and never committed.
set -euo pipefail
REF_DIR=${REF_DIR:?set REF_DIR to the reference checkout}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
if [ ! -f "$REF_DIR/src/advection.cpp" ]; then
  echo "build_ref.sh: reference sources not found under $REF_DIR" >&2
  exit 3
fi
mkdir -p "$OUT/obj_exact" "$OUT/obj_fast"
sed -n '1,559p;742,1016p' "$REF_DIR/src/shape_optimization.cpp" > "$OUT/shape_optimization_noeigen.cpp"
echo '}  // namespace navier_stokes' >> "$OUT/shape_optimization_noeigen.cpp"
SRCS=""
for s in advection diffusion boundary compute mesh utils params init; do SRCS="$SRCS $REF_DIR/src/$s.cpp"; done
SRCS="$SRCS $OUT/shape_optimization_noeigen.cpp $HERE/ref_harness.cpp"
INC="-I$HERE/shims -I$REF_DIR/include -include iomanip -include array -include numeric -include algorithm -include limits -include cmath"
build() {
  local flavour=$1; shift
  local objs="" pids=""
  for src in $SRCS; do
    local o="$OUT/obj_$flavour/$(basename "${src%.cpp}").o"
    g++ -std=c++17 -fopenmp -w "$@" $INC -c "$src" -o "$o" &
    pids="$pids $!"
    objs="$objs $o"
  done
  for p in $pids; do wait "$p"; done
  g++ -fopenmp $objs -o "$OUT/o2f_ref_$flavour"
}
build exact -O2 -ffp-contract=off
build fast -O3 -march=x86-64-v3
# The link check of the drop-in adapter: the reference's exact objects (its
# own harness left out), the adapter under another namespace, libo2f.so.
PKG=$(cd "$HERE/../optimisation2forme_b200" && pwd)
if [ -f "$PKG/libo2f.so" ]; then
  g++ -std=c++17 -fopenmp -w -O2 -ffp-contract=off -DO2F_ADAPTER_NS=o2f_adapter $INC -I"$HERE/../include" \
    -c "$PKG/adapters/navier_stokes_o2f.cpp" -o "$OUT/obj_exact/adapter_o2f.o"
  g++ -std=c++17 -fopenmp -w -O2 -ffp-contract=off $INC -c "$HERE/adapter_check.cpp" -o "$OUT/obj_exact/adapter_check.o"
  REFOBJS=""
  for s in advection diffusion boundary compute mesh utils params init shape_optimization_noeigen; do
    REFOBJS="$REFOBJS $OUT/obj_exact/$s.o"
  done
  g++ -fopenmp $REFOBJS "$OUT/obj_exact/adapter_o2f.o" "$OUT/obj_exact/adapter_check.o" -L"$PKG" -lo2f \
    -Wl,-rpath,'$ORIGIN/../../optimisation2forme_b200' -o "$OUT/o2f_adapter_check"
fi
echo "built $OUT/o2f_ref_exact $OUT/o2f_ref_fast"
