#!/usr/bin/env bash
# Builds oracle/_ref/ref_gpu_program: the reference's own GPU solver
# (Solver_gpu.cu and its kernel files, unmodified, compiled for sm_100a with
# relocatable device code as the reference's makefile does, -maxrregcount=128)
# behind the program set-up of oracle/ref_program.cpp.  Test and bench
# infrastructure only (the reference GPU baseline): sources are read where they
# lie, outputs go to oracle/_ref/gpu/.
# Usage: oracle/build_ref_gpu.sh [REFERENCE_DIR]
#   (default: $LBFS_REFERENCE_DIR, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${LBFS_REFERENCE_DIR:-/root/reference}}"
OUT="$HERE/_ref/gpu"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ ! -f "$REF/Solver_gpu.cu" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref/ref_gpu_program" >&2
  exit 0
fi
mkdir -p "$OUT"
INC="-I$HERE/ref_stub_gpu -I$REF -I/usr/local/cuda/include"
HOST_SRC="unstructured_mesh Mesh global_variables domain_geometry initial_conditions vector_var gradients
          Boundary_Conditions Solution unstructured_bcs lagrangian_object tecplot_output quad_bcs quad_bcs_plus
          post_processing residuals flux_var RungeKutta external_forces preprocessor tinyxml2"
CU_SRC="Solver_gpu LBFS immersed_boundary_method spring_network common_kernels wlc"
pids=()
for f in $HOST_SRC; do
  g++ -std=c++17 -O2 -fpermissive -w $INC -c "$REF/$f.cpp" -o "$OUT/$f.o" & pids+=($!)
done
for f in $CU_SRC; do
  "$NVCC" -std=c++17 -O2 -rdc=true -gencode arch=compute_100a,code=sm_100a -maxrregcount=128 -w $INC \
      -c "$REF/$f.cu" -o "$OUT/$f.o" & pids+=($!)
done
g++ -std=c++17 -O2 -fpermissive -w $INC -DREF_GPU_PROGRAM -c "$HERE/ref_program.cpp" -o "$OUT/ref_program.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
OBJ=""
for f in $HOST_SRC $CU_SRC ref_program; do OBJ="$OBJ $OUT/$f.o"; done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$HERE/_ref/ref_gpu_program" $OBJ -lcudart
echo "built $HERE/_ref/ref_gpu_program"
