#!/usr/bin/env bash
# Builds the drop-in IPlanarRouteBackend shim against the reference's headers:
#   apgar_b200/adapter/_build/b200_planar_backend.o   the shim (what a
#                                                     reference build links in
#                                                     place of its CUDA unit)
#   apgar_b200/adapter/_build/adapter_check           GPU check of the shim
#                                                     over the golden fixtures
#                                                     (test infrastructure;
#                                                     links the reference's CPU
#                                                     objects from oracle/_ref)
#   apgar_b200/adapter/_build/prepared_batch_check    GPU check through the
#                                                     reference's own prepared
#                                                     host path, built from a
#                                                     patched copy of the
#                                                     reference (below)
#   apgar_b200/adapter/_build/dropin_bench            the drop-in benchmark on the
#                                                     reference corpus (bench.py
#                                                     --workload dropin)
# The patched copy: reference_generator.patch (the B200 persistent generators
# and their descriptor, the change a maintainer applies to the reference) is
# applied to copies of the files it touches under _build/ref_patched/, and
# every reference source the checks need is compiled against that tree.  The
# reference tree itself is only read.
# Needs the reference tree (APGAR_REFERENCE, or the tree oracle/build_ref.sh
# recorded), g++ with C++20, patch, libapgar_b200.so and
# oracle/_ref/libapgar_ref.a (oracle/build_ref.sh).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/../.." && pwd)"
REF="${APGAR_REFERENCE:-$(cat "$ROOT/oracle/_ref/reference_root.txt" 2>/dev/null || echo /root/reference)}"
OUT="$HERE/_build"
CXX="${CXX:-g++}"
FLAGS=(-std=c++20 -O2 -Wall -Wextra -fPIC -I"$REF/include" -I"$REF" -I"$ROOT/include")
mkdir -p "$OUT"
"$CXX" "${FLAGS[@]}" -c "$HERE/b200_planar_backend.cc" -o "$OUT/b200_planar_backend.o"
if [ "${1:-}" = "--check" ]; then
  echo "$OUT/b200_planar_backend.o"
  exit 0
fi
"$CXX" "${FLAGS[@]}" "$ROOT/tests/native/adapter_check.cc" "$OUT/b200_planar_backend.o" \
  "$ROOT/oracle/_ref/libapgar_ref.a" -L"$ROOT/apgar_b200" -lapgar_b200 \
  -Wl,-rpath,'$ORIGIN/../..' -o "$OUT/adapter_check"
echo "$OUT/adapter_check"

# ---- the reference with the generator patch applied ----
PATCHED="$OUT/ref_patched"
PATCHED_FILES=(include/apgar/gpu/planar_router.h src/gpu/planar_router.cc
               src/candidates/gpu_candidate_adapter.cc)
rm -rf "$PATCHED"
for f in "${PATCHED_FILES[@]}"; do
  mkdir -p "$PATCHED/$(dirname "$f")"
  cp "$REF/$f" "$PATCHED/$f"
done
(cd "$PATCHED" && patch -p1 -s --no-backup-if-mismatch < "$HERE/reference_generator.patch")
PFLAGS=(-std=c++20 -O2 -fPIC -I"$PATCHED/include" -I"$REF/include" -I"$REF")
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
  src/candidates/route_candidate.cc
  src/candidates/gpu_candidate_adapter.cc
)
mkdir -p "$PATCHED/obj"
OBJS=()
PIDS=()
for src in "${SRCS[@]}"; do
  in="$REF/$src"
  [ -f "$PATCHED/$src" ] && in="$PATCHED/$src"
  obj="$PATCHED/obj/$(echo "$src" | tr '/' '_' | sed 's/\.cc$/.o/')"
  "$CXX" "${PFLAGS[@]}" -c "$in" -o "$obj" &
  PIDS+=($!)
  OBJS+=("$obj")
done
for pid in "${PIDS[@]}"; do wait "$pid"; done  # each compile's own status
rm -f "$PATCHED/libapgar_ref_patched.a"
ar rcs "$PATCHED/libapgar_ref_patched.a" "${OBJS[@]}"
"$CXX" "${PFLAGS[@]}" -Wall -Wextra -I"$ROOT/include" -c "$HERE/b200_planar_backend.cc" \
  -o "$PATCHED/b200_planar_backend.o"
"$CXX" "${PFLAGS[@]}" -Wall -Wextra -c "$HERE/fault_injecting_backend.cc" \
  -o "$PATCHED/fault_injecting_backend.o"
# the KiCad fixture's text, for the corpus the check builds on the GPU box
python3 - "$REF/tests/fixtures/m1_exactness.kicad_pcb" "$PATCHED/kicad_fixture.cc" <<'PY'
import sys
data = open(sys.argv[1], "rb").read()
body = ",".join(str(b) for b in data)
with open(sys.argv[2], "w") as f:
    f.write("extern const char kKicadFixture[] = {%s};\n" % body)
    f.write("extern const unsigned long kKicadFixtureSize = %d;\n" % len(data))
PY
"$CXX" "${PFLAGS[@]}" -Wall -Wextra "$ROOT/tests/native/prepared_batch_check.cc" \
  "$PATCHED/kicad_fixture.cc" "$PATCHED/b200_planar_backend.o" "$PATCHED/fault_injecting_backend.o" \
  "$PATCHED/libapgar_ref_patched.a" -L"$ROOT/apgar_b200" -lapgar_b200 -lpthread \
  -Wl,-rpath,'$ORIGIN/../..' -o "$OUT/prepared_batch_check"
echo "$OUT/prepared_batch_check"
# the drop-in benchmark on the reference's corpus (bench.py --workload dropin)
"$CXX" "${PFLAGS[@]}" -Wall -Wextra "$HERE/dropin_bench.cc" "$PATCHED/kicad_fixture.cc" \
  "$PATCHED/b200_planar_backend.o" "$PATCHED/libapgar_ref_patched.a" -L"$ROOT/apgar_b200" \
  -lapgar_b200 -lpthread -Wl,-rpath,'$ORIGIN/../..' -o "$OUT/dropin_bench"
echo "$OUT/dropin_bench"
