#!/usr/bin/env bash
# Builds the reference's CPU path from its own sources (read in place, never
# copied into this repository) into oracle/_ref/:
#   oracle/_ref/libapgar_ref.a   board IR, geometry, geometry compiler, routing
#                                (CPU A*), device-view flattening, host GPU
#                                dispatch/validation, corpus + KiCad adapter
#   oracle/_ref/ref_fixtures     driver that writes tests/golden fixtures
#   oracle/_ref/ref_lattice      compile + CPU A* on box-obstacle lattices
# TEST INFRASTRUCTURE ONLY.  Needs the reference tree (REF, default
# /root/reference) and g++ with C++20; the GPU box only uses prebuilt outputs.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${APGAR_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
CXX="${CXX:-g++}"
FLAGS=(-std=c++20 -O2 -fPIC -I"$REF/include" -I"$REF")
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OUT/obj"
SRCS=(
  src/board_ir/board.cc
  src/geometry/exact.cc
  src/geometry_compiler/compiled_board.cc
  src/routing/candidate_policy.cc
  src/routing/planar_route.cc
  src/routing/cpu_astar.cc
  src/gpu/device_board.cc
  src/gpu/planar_router.cc
  src/adapters/kicad_fixture.cc
  src/benchmark/planar_corpus.cc
  src/allocator/resource_accounting.cc
  src/allocator/negotiated_regeneration_plan.cc
  src/allocator/cpu_sequential_negotiated_routing.cc
)
OBJS=()
for src in "${SRCS[@]}"; do
  obj="$OUT/obj/$(echo "$src" | tr '/' '_' | sed 's/\.cc$/.o/')"
  if [ ! -f "$obj" ] || [ "$REF/$src" -nt "$obj" ]; then
    "$CXX" "${FLAGS[@]}" -c "$REF/$src" -o "$obj"
  fi
  OBJS+=("$obj")
done
rm -f "$OUT/libapgar_ref.a"
ar rcs "$OUT/libapgar_ref.a" "${OBJS[@]}"
"$CXX" "${FLAGS[@]}" "$HERE/ref_fixtures.cc" "$OUT/libapgar_ref.a" -o "$OUT/ref_fixtures"
"$CXX" "${FLAGS[@]}" "$HERE/ref_lattice.cc" "$OUT/libapgar_ref.a" -o "$OUT/ref_lattice"
# where the checker was built from, for the tests that read reference files
(cd "$REF" && pwd) > "$OUT/reference_root.txt"
echo "$OUT"
