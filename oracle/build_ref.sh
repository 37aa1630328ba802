#!/bin/sh
# Builds the reference pdMTEL solver from its own C++ sources, where they lie,
# into oracle/_ref/ (git-ignored).  The result is test infrastructure only: the
# reference harness that produces golden vectors and the timed CPU baseline.
#
#   sh oracle/build_ref.sh REFERENCE_DIR     (or PDMTEL_REFERENCE=REFERENCE_DIR)
#
# The shipped reference does not compile as-is under g++ 13; three minimal
# patches are applied to a scratch copy under oracle/_ref/src (never committed):
#   1. pdGauss.h lacks the MLS coefficient accessors SetCoeff/GetCoeff that
#      pdDataManager2.cpp:245 and pdDataManager.cpp:2445 call; they are added.
#   2. pdDataManager3.cpp:23 needs `typename` before a dependent iterator type.
#   3. <cstring>/<cmath> are force-included (memset at pdDataManager2.cpp:1588).
# main.cpp (windows.h), pdHandle.cpp (#included by pdDataManager.h), the dead
# pdBCTract.cpp / pdBCVelocTime.cpp and debug_new.cpp are not compiled.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${PDMTEL_REFERENCE:-}}
if [ -z "$REF" ]; then
    echo "build_ref.sh: give the reference source folder as the first argument or PDMTEL_REFERENCE" >&2
    exit 2
fi
OUT="$HERE/_ref"
if [ ! -f "$REF/pdDataManager.cpp" ]; then
    echo "build_ref.sh: reference sources not found at $REF" >&2
    exit 2
fi
mkdir -p "$OUT/src" "$OUT/obj"
for f in "$REF"/*.cpp "$REF"/*.h; do
    cp "$f" "$OUT/src/"
done
chmod u+w "$OUT"/src/*

# patch 1: MLS coefficient accessors on pdGauss
if ! grep -q "GetCoeff" "$OUT/src/pdGauss.h"; then
    sed -i 's/^#include "pdIntgPoint.h"/#include "pdIntgPoint.h"\nclass pdVector;/' "$OUT/src/pdGauss.h"
    sed -i 's/^\tdouble GetWeightX3() const;/\tdouble GetWeightX3() const;\n\tvoid SetCoeff(pdVector* c) { _coeff = c; }\n\tpdVector* GetCoeff() const { return _coeff; }/' "$OUT/src/pdGauss.h"
    sed -i 's/^\tdouble _weightX1, _weightX2, _weightX3;/\tdouble _weightX1, _weightX2, _weightX3;\n\tpdVector* _coeff = 0;/' "$OUT/src/pdGauss.h"
fi
# patch 2: dependent type name
sed -i 's/^\tfor (vector<T\*>::iterator itor=vec.begin()/\tfor (typename vector<T*>::iterator itor=vec.begin()/' "$OUT/src/pdDataManager3.cpp"

CXX=${CXX:-g++}
# -ffp-contract=off keeps every multiply and add separately rounded, as the
# reference's own (SSE2, no FMA) x86-64 build does.
CXXFLAGS="-O2 -std=c++17 -fpermissive -w -ffp-contract=off -include cstring -include cmath"
OBJS=""
for f in "$OUT"/src/*.cpp; do
    b=$(basename "$f" .cpp)
    case "$b" in
        main|pdHandle|pdBCTract|pdBCVelocTime|debug_new) continue ;;
    esac
    o="$OUT/obj/$b.o"
    if [ ! -f "$o" ] || [ "$f" -nt "$o" ]; then
        $CXX $CXXFLAGS -I"$OUT/src" -c "$f" -o "$o" &
    fi
    OBJS="$OBJS $o"
done
wait
$CXX $CXXFLAGS -I"$OUT/src" -c "$HERE/ref_harness.cpp" -o "$OUT/obj/ref_harness.o"
$CXX -O2 -o "$OUT/pdref_harness" "$OUT/obj/ref_harness.o" $OBJS
echo "built $OUT/pdref_harness"
