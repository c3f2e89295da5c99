#!/usr/bin/env bash
# Builds oracle/_ref/libref_lbfs.so from the reference sources where they lie
# (read-only), with the host stubs in oracle/ref_stub/ and the driver
# oracle/ref_driver.cpp.  Test infrastructure only: it produces the golden
# vectors under tests/golden/ and the CPU timing of bench.py's reference arm.
# Usage: oracle/build_ref.sh [REFERENCE_DIR]
#   (default: $LBFS_REFERENCE_DIR, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${LBFS_REFERENCE_DIR:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -f "$REF/LBFS.cu" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT"
# -ffp-contract=off keeps each multiply and add separately rounded, as the
# reference's own CPU build does; -O2 as in the reference makefile.
CXXFLAGS="-std=c++17 -O2 -ffp-contract=off -fPIC -fpermissive -w -I$HERE/ref_stub -I$REF"
HOST_SRC="unstructured_mesh Mesh global_variables domain_geometry initial_conditions vector_var gradients
          Boundary_Conditions Solution unstructured_bcs lagrangian_object tecplot_output quad_bcs quad_bcs_plus
          post_processing residuals flux_var RungeKutta external_forces"
KERNEL_SRC="LBFS immersed_boundary_method spring_network common_kernels"
pids=()
for f in $HOST_SRC; do
  g++ $CXXFLAGS -c "$REF/$f.cpp" -o "$OUT/$f.o" & pids+=($!)
done
for f in $KERNEL_SRC; do
  g++ $CXXFLAGS -x c++ -c "$REF/$f.cu" -o "$OUT/$f.o" & pids+=($!)
done
g++ $CXXFLAGS -c "$HERE/ref_driver.cpp" -o "$OUT/ref_driver.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
g++ -shared -o "$OUT/libref_lbfs.so" "$OUT"/*.o
echo "built $OUT/libref_lbfs.so"
