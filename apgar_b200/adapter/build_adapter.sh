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
# Needs the reference tree (APGAR_REFERENCE, default /root/reference), g++ with
# C++20, libapgar_b200.so and oracle/_ref/libapgar_ref.a (oracle/build_ref.sh).
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
