#!/usr/bin/env bash
# Test infrastructure only: compiles the reference's own GMRES-FMM BVP sources (read
# in place under the reference checkout) into oracle/_ref/, for pinning the oracle.
#   1. regenerates the three missing AAA_*_FMM.hpp tables (gen_aaa_tables.cpp),
#   2. derives BEM_solveBVP.hpp with the compile-time expansion order set to P
#      (the reference hard-codes 10 at bem/BEM_solveBVP.hpp:563),
#   3. compiles ref_harness.cpp + lib/src/*.cpp with g++ (no CMake).
# Outputs only into oracle/_ref/ (git-ignored).  Usage: build_ref.sh [P ...]
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${BEM_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/../_ref"
ORDERS=("$@")
[ ${#ORDERS[@]} -eq 0 ] && ORDERS=(8 10)
if [ ! -d "$REF/bem" ]; then echo "reference checkout not found at $REF" >&2; exit 3; fi
mkdir -p "$OUT/gen/include"
g++ -O1 -std=gnu++20 -o "$OUT/gen/gen_aaa_tables" "$HERE/gen_aaa_tables.cpp" -lquadmath
"$OUT/gen/gen_aaa_tables" "$OUT/gen/include" 12
for P in "${ORDERS[@]}"; do
  mkdir -p "$OUT/gen/p$P"
  sed -E "s#(Buckets<std::shared_ptr<source4FMM<target4FMM>>, )10( /\*)#\1$P\2#" "$REF/bem/BEM_solveBVP.hpp" > "$OUT/gen/p$P/BEM_solveBVP.hpp"
  grep -q "target4FMM>>, $P " "$OUT/gen/p$P/BEM_solveBVP.hpp" || { echo "order patch failed" >&2; exit 4; }
  g++ -std=gnu++23 -O3 -march=x86-64-v3 -fopenmp -w \
      -I"$OUT/gen/p$P" -I"$OUT/gen/include" -I"$REF/bem" -I"$REF/lib/include" \
      "$HERE/ref_harness.cpp" "$HERE/lapack_shim.cpp" "$REF"/lib/src/Network.cpp "$REF"/lib/src/networkPoint.cpp "$REF"/lib/src/networkLine.cpp \
      "$REF"/lib/src/networkFace.cpp "$REF"/lib/src/networkTetra.cpp \
      -o "$OUT/bem_ref_p$P" -lquadmath
  echo "built $OUT/bem_ref_p$P"
done
