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
          post_processing residuals flux_var RungeKutta external_forces preprocessor tinyxml2"
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
KERNEL_OBJ=""
for f in $KERNEL_SRC; do KERNEL_OBJ="$KERNEL_OBJ $OUT/$f.o"; done
HOST_OBJ=""
for f in $HOST_SRC; do HOST_OBJ="$HOST_OBJ $OUT/$f.o"; done
g++ -shared -o "$OUT/libref_lbfs.so" $HOST_OBJ $KERNEL_OBJ "$OUT/ref_driver.o"
echo "built $OUT/libref_lbfs.so"

# The drop-in program: the reference's own set-up (XML deck, preprocessor, mesh,
# boundary conditions, lagrangian object; oracle/ref_program.cpp after
# program::run) calling gpu_solver::General_Purpose_Solver_mk_i as linked from
# the repository's drop-in (integration/Solver_gpu_lbfs.cpp) over liblbfs_b200.so
# instead of the reference's Solver_gpu.cu.  Needs the library built first.
ROOT="$(dirname "$HERE")"
LIBDIR="$ROOT/lbfs-ibm-ade-sp_b200/lbfs_b200/_lib"
if [ -f "$LIBDIR/liblbfs_b200.so" ]; then
  mkdir -p "$OUT/dropin"
  g++ $CXXFLAGS -I"$ROOT/include" -c "$HERE/ref_program.cpp" -o "$OUT/dropin/ref_program.o" &
  p1=$!
  g++ $CXXFLAGS -I"$ROOT/include" -c "$ROOT/lbfs-ibm-ade-sp_b200/integration/Solver_gpu_lbfs.cpp" \
      -o "$OUT/dropin/Solver_gpu_lbfs.o" &
  p2=$!
  wait $p1; wait $p2
  g++ -o "$OUT/dropin_program" "$OUT/dropin/ref_program.o" "$OUT/dropin/Solver_gpu_lbfs.o" $HOST_OBJ \
      -L"$LIBDIR" -llbfs_b200 -Wl,-rpath,'$ORIGIN/../../lbfs-ibm-ade-sp_b200/lbfs_b200/_lib'
  echo "built $OUT/dropin_program"
else
  echo "liblbfs_b200.so not built yet; skipping oracle/_ref/dropin_program" >&2
fi

# The reference's CPU solver behind the same set-up (Solver::General_Purpose_Solver_mk_i,
# the BASELINE's CPU row): ref_program.cpp built with REF_CPU_SOLVER.
mkdir -p "$OUT/cpu"
g++ $CXXFLAGS -c "$REF/Solver.cpp" -o "$OUT/cpu/Solver.o" &
p1=$!
g++ $CXXFLAGS -DREF_CPU_SOLVER -c "$HERE/ref_program.cpp" -o "$OUT/cpu/ref_program.o" &
p2=$!
wait $p1; wait $p2
g++ -o "$OUT/ref_cpu_program" "$OUT/cpu/ref_program.o" "$OUT/cpu/Solver.o" $HOST_OBJ
echo "built $OUT/ref_cpu_program"
