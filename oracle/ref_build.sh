#!/usr/bin/env bash
# Builds the reference engine (PS_AGONY2D, C++20/23, AVX2) as a CPU oracle and timed CPU baseline.
#
# Test infrastructure only: the product never links or loads anything built here.
#
# The reference is MSVC code. Five small portability patches are needed for g++ 13; they are applied
# to a throw-away copy of the engine tree under oracle/_ref/src (git-ignored), never to the original:
#   1. Integration/Integrator.cpp:7      a stray token after an #include directive is removed.
#   2. Narrow/NarrowPhaseCollisionDetector.h:30-34  anonymous union over the non-trivial Handle (an MSVC
#      extension) becomes two plain Handle members; the dense-index view of the union is replaced by
#      Handle::slot, which is what the union aliased (.h:54-55 write it, .cpp:703-704 read it).
#   3. Missing standard includes are forced with -include (cstring, cstdint, span, xmmintrin.h).
#   4. __forceinline (MSVC) is mapped to the GCC always_inline attribute.
#   5. CollisionMethods/PolygonCapsule.cpp: its `goto nextPair` jumps over initialisations (a GCC error). The
#      statements from the side-axis test to the label are wrapped in one block, so the jumps cross a whole
#      block instead; nothing else changes (same statements, same order, same arithmetic).
# Tracy's header is included unconditionally by Profiling/TracyProfiler.h:2; an empty stub stands in.
#
# Flags are the parity build: -O2 -mavx2 -mfma -ffp-contract=off (no fast-math). Explicit FMA intrinsics in
# the reference's SIMD wrapper still fuse; that is the reference's own arithmetic.
#
# Usage: oracle/ref_build.sh [reference_root]. The reference root is the argument, else $AG2D_REFERENCE_ROOT, else
# /root/reference (the build container's checkout). Output: oracle/_ref/libagony_ref.so. Exit status 2: no
# reference checkout there (nothing built).
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${1:-${AG2D_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
SRC_ENGINE="$REF_ROOT/PhysicsSimulation-Agony/PS_AGONY2D"
LIB_INC="$REF_ROOT/Libraries/include"

if [ ! -d "$SRC_ENGINE" ]; then
  echo "ref_build: reference engine not found at $SRC_ENGINE" >&2
  exit 2
fi

mkdir -p "$OUT/src" "$OUT/obj" "$OUT/stub/tracy"
rm -rf "$OUT/src/PS_AGONY2D"
cp -r "$SRC_ENGINE" "$OUT/src/PS_AGONY2D"
chmod -R u+w "$OUT/src/PS_AGONY2D"
: > "$OUT/stub/tracy/Tracy.hpp"

E="$OUT/src/PS_AGONY2D"
# Patch 1.
sed -i 's|#include "PS_AGONY2D/FastCosSin.h"RealSimd::storeu|#include "PS_AGONY2D/FastCosSin.h"|' "$E/Integration/Integrator.cpp"
# Patch 2 (header): replace the anonymous union block by two Handle members.
python3 - "$E/CollisionDetection/Narrow/NarrowPhaseCollisionDetector.h" "$E/CollisionDetection/Narrow/NarrowPhaseCollisionDetector.cpp" <<'PY'
import re, sys
h, c = sys.argv[1], sys.argv[2]
s = open(h, encoding="utf-8-sig").read()
s2 = re.sub(r"union\s*\{\s*struct\s*\{\s*Handle colliderA, colliderB;\s*\};\s*struct\s*\{[^}]*\};\s*\};",
            "Handle colliderA, colliderB;", s, count=1)
assert s2 != s, "union patch did not apply"
s2 = s2.replace("indexA = colliderIndexA;", "colliderA.slot = colliderIndexA;")
s2 = s2.replace("indexB = colliderIndexB;", "colliderB.slot = colliderIndexB;")
open(h, "w").write(s2)
t = open(c, encoding="utf-8-sig").read()
t2 = t.replace("const ObjectDenseIndex indexA = d.indexA;", "const ObjectDenseIndex indexA = d.colliderA.slot;")
t2 = t2.replace("const ObjectDenseIndex indexB = d.indexB;", "const ObjectDenseIndex indexB = d.colliderB.slot;")
assert t2 != t, "finalizeResults patch did not apply"
open(c, "w").write(t2)
PY
# Patch 5: PolygonCapsule.cpp, the block around the code the goto jumps over.
python3 - "$E/CollisionDetection/Narrow/CollisionMethods/PolygonCapsule.cpp" <<'PY'
import sys
p = sys.argv[1]
s = open(p, encoding="utf-8-sig").read()
a = "            const Real sideOffset = glm::dot(sideAxis, centerLocal);"
b = "            nextPair:\n"
assert s.count(a) == 1 and s.count(b) == 1, "PolygonCapsule patch did not apply"
s = s.replace(a, "            {\n" + a).replace(b, "            }\n            nextPair:;\n")
open(p, "w").write(s)
PY

CXX="${CXX:-g++}"
FLAGS=(-std=c++23 -O2 -mavx2 -mfma -ffp-contract=off -fPIC -fpermissive -Wno-interference-size -w
       -include cstring -include cstdint -include span -include xmmintrin.h
       "-D__forceinline=__attribute__((always_inline))"
       -I"$OUT/src" -I"$LIB_INC" -I"$OUT/stub")

mapfile -t SOURCES < <(cd "$E" && find . -name '*.cpp' | sort)
pids=()
objs=()
for s in "${SOURCES[@]}"; do
  o="$OUT/obj/$(echo "$s" | sed 's|^\./||; s|/|_|g; s|\.cpp$|.o|')"
  objs+=("$o")
  "$CXX" "${FLAGS[@]}" -c "$E/$s" -o "$o" &
  pids+=($!)
  if [ "${#pids[@]}" -ge 8 ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
done
for p in "${pids[@]}"; do wait "$p"; done

# The harness reaches private members of Simulation (phase-by-phase taps) with -fno-access-control.
"$CXX" "${FLAGS[@]}" -fno-access-control -c "$HERE/ref_harness.cpp" -o "$OUT/obj/ref_harness.o"
"$CXX" -shared -o "$OUT/libagony_ref.so" "${objs[@]}" "$OUT/obj/ref_harness.o" -lpthread
echo "ref_build: built $OUT/libagony_ref.so"
