#!/bin/sh
# Compile the reference's Tier-1 block decoder where it lies (no copies) together with
# oracle/ref_t1_driver.cpp into oracle/_ref/libref_t1.so.  Needs the reference tree
# (argument or J2K_REFERENCE_DIR); the shared object is git-ignored and travels with the repo.
set -e
REF=${1:-$J2K_REFERENCE_DIR}
[ -n "$REF" ] || { echo "usage: $0 <reference root> (or set J2K_REFERENCE_DIR)" >&2; exit 2; }
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
D="$REF/decoder"
[ -d "$D/codec/src" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
INC="-I$D/codec/include -I$D/common/include -I$D/tools/include -I$D/core/include -I$D/codec/src"
FLAGS="-O2 -w -fPIC -include $HERE/ref_prelude.h"
g++ $FLAGS $INC -c "$D/codec/src/bmi_block_decoder.cpp" -o "$OUT/bmi_block_decoder.o"
g++ $FLAGS $INC -c "$D/codec/src/bmi_mq_decoder.cpp" -o "$OUT/bmi_mq_decoder.o"
g++ $FLAGS $INC -c "$HERE/ref_t1_driver.cpp" -o "$OUT/ref_t1_driver.o"
g++ -shared -o "$OUT/libref_t1.so" "$OUT/ref_t1_driver.o" "$OUT/bmi_block_decoder.o" "$OUT/bmi_mq_decoder.o"
rm -f "$OUT"/*.o
echo "built $OUT/libref_t1.so"
