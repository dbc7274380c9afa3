#!/bin/bash
# Test infrastructure: builds the reference OPS library and the reference
# OpenMP apps from the read-only reference checkout into oracle/_ref
# (git-ignored; it travels to the GPU host with the working tree).
#
# Recipe (no reference build system is run):
#   1. libops_seq.a from the nine sources the reference's `seq` target lists
#      (ops/c/Makefile:221-223), compiled with the reference's gnu flags
#      (makefiles/Makefile.gnu: -O3 -fPIC -ffloat-store -std=c++11 -fopenmp).
#   2. Per app: the app sources are copied into oracle/_ref/<app>/ (the
#      reference's legacy translator writes next to its inputs), translated
#      with ops_translator_legacy/c/ops.py, and compiled as the reference's
#      `<app>_openmp` target does (makefiles/Makefile.c_app:218-224), plus the
#      oracle hook object (full-precision printing, optional field dumps).
#
# usage: oracle/build_ref.sh [reference_root]   (default: $OPS_REFERENCE_ROOT)
set -euo pipefail
REF=${1:-${OPS_REFERENCE_ROOT:-}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
# /usr/bin/g++ carries the OpenMP spec file; another g++ earlier on PATH may not
CXX=${OPS_ORACLE_CXX:-$( [ -x /usr/bin/g++ ] && echo /usr/bin/g++ || echo g++ )}
CXXFLAGS="-O3 -fPIC -ffloat-store -std=c++11 -fopenmp -Dgnu -w"
INC="-I$REF/ops/c/include"

if [ ! -d "$REF/ops/c/src" ]; then
  echo "reference tree not found at $REF" >&2
  exit 1
fi
mkdir -p "$OUT/obj" "$OUT/lib" "$OUT/bin"

# ---- 1. reference runtime library ------------------------------------------
LIBSRC="core/ops_lib_core core/ops_instance core/ops_lazy externlib/ops_checkpointing
        externlib/ops_util sequential/ops_host_common sequential/ops_host_singlenode
        core/ops_dummy_singlenode externlib/ops_checkpointing_strategy"
objs=()
for s in $LIBSRC; do
  o="$OUT/obj/$(basename "$s").o"
  if [ ! -f "$o" ] || [ "$REF/ops/c/src/$s.cpp" -nt "$o" ]; then
    $CXX $CXXFLAGS $INC -c "$REF/ops/c/src/$s.cpp" -o "$o" &
  fi
  objs+=("$o")
done
wait
rm -f "$OUT/lib/libops_seq.a"
ar rcs "$OUT/lib/libops_seq.a" "${objs[@]}"
$CXX $CXXFLAGS $INC -c "$HERE/ref_drivers/oracle_hooks.cpp" -o "$OUT/obj/oracle_hooks.o"

# ---- 2. apps -----------------------------------------------------------------
# build_app <name> <srcdir> "<ops files>" "<other files>" "<extra files to copy>"
build_app() {
  local name=$1 src=$2 opsf=$3 other=$4 extra=$5
  local dir="$OUT/$name"
  mkdir -p "$dir"
  cp "$src"/*.h "$dir"/ 2>/dev/null || true
  cp "$src"/*.cpp "$dir"/ 2>/dev/null || true
  for e in $extra; do cp "$e" "$dir"/; done
  (cd "$dir" && python3 "$REF/ops_translator_legacy/c/ops.py" $opsf > translate.log 2>&1)
  local gen=()
  for f in $opsf; do gen+=("${f%.cpp}_ops.cpp"); done
  (cd "$dir" && $CXX $CXXFLAGS $INC -I. -include "$HERE/ref_drivers/fullprec_hook.h" \
      "${gen[@]}" $other mpi_openmp/mpi_openmp_kernels.cpp "$OUT/obj/oracle_hooks.o" \
      -L"$OUT/lib" -lops_seq -o "$OUT/bin/$name")
  echo "built $OUT/bin/$name"
}

LAP=$REF/apps/c/laplace2d_tutorial/step7
build_app laplace2d_step7 "$LAP" "laplace2d.cpp" "" "" &
SEEDED=$OUT/laplace2d_seeded_src
mkdir -p "$SEEDED"
cp "$LAP/laplace_kernels.h" "$SEEDED/"
cp "$HERE/ref_drivers/laplace_seeded.cpp" "$HERE/src/seeded_rng.h" "$SEEDED/"
build_app laplace2d_seeded "$SEEDED" "laplace_seeded.cpp" "" "" &

CL=$REF/apps/c/CloverLeaf
build_app cloverleaf "$CL" \
  "clover_leaf.cpp initialise_chunk.cpp generate.cpp ideal_gas.cpp update_halo.cpp field_summary.cpp viscosity.cpp calc_dt.cpp PdV.cpp revert.cpp accelerate.cpp flux_calc.cpp advec_cell.cpp advec_mom.cpp reset_field.cpp" \
  "start.cpp time_step.cpp build_field.cpp read_input.cpp initialise.cpp advection.cpp" "" &

CL3=$REF/apps/c/CloverLeaf_3D
build_app cloverleaf3d "$CL3" \
  "clover_leaf.cpp initialise_chunk.cpp generate.cpp ideal_gas.cpp update_halo.cpp field_summary.cpp viscosity.cpp calc_dt.cpp PdV.cpp revert.cpp accelerate.cpp flux_calc.cpp advec_cell.cpp advec_mom.cpp reset_field.cpp" \
  "start.cpp time_step.cpp build_field.cpp read_input.cpp initialise.cpp advection.cpp" "" &

# halo transfer cases: a driver of our own on the reference's public API,
# compiled against libops_seq.a with the reference's template loop path
# (ops_seq_v2.h, no translation)
(mkdir -p "$OUT/halo_cases" && cd "$OUT/halo_cases" && \
  $CXX $CXXFLAGS $INC "$HERE/ref_drivers/halo_cases.cpp" -L"$OUT/lib" -lops_seq -o "$OUT/bin/halo_cases" && \
  echo "built $OUT/bin/halo_cases") &

TL=$REF/apps/c/TeaLeaf
build_app tealeaf "$TL" \
  "tea_leaf.cpp field_summary.cpp generate.cpp initialise_chunk.cpp start.cpp set_field.cpp tea_leaf_cg.cpp tea_leaf_cheby.cpp tea_leaf_common.cpp tea_leaf_jacobi.cpp tea_leaf_ppcg.cpp update_halo.cpp" \
  "$(cd "$TL" && ls *.cpp | grep -v -E '^(tea_leaf|field_summary|generate|initialise_chunk|start|set_field|tea_leaf_cg|tea_leaf_cheby|tea_leaf_common|tea_leaf_jacobi|tea_leaf_ppcg|update_halo)\.cpp$' | tr '\n' ' ')" "" &
wait
ls -la "$OUT/bin"
