#!/bin/sh
# Build the reference's whole CPU decoder (host Tier-2, C++ Tier-1 on worker threads, CPU
# inverse DWT / MCT, BMI::Decoder engine) from its sources where they lie, into
# oracle/_ref/libref_cpu.so, behind the small C entry points of oracle/ref_cpu_driver.cpp.
# TEST AND BASELINE INFRASTRUCTURE ONLY: the tests use it to pin the oracle and the device
# path to the reference's own output, and bench.py's CPU arm times it.
#
# Usage: oracle/build_ref_cpu.sh <reference root>   (or J2K_REFERENCE_DIR=<root>)
#
# The reference targets 32-bit x86 and a CUDA-1.0 GPU back end; on x86-64 with CUDA 12 its
# CPU path needs these adjustments, none of which edits a file under the reference root:
#   * codec.h (decoder/codec/include/codec.h) is shadowed by a generated copy in
#     oracle/_ref/shim with three lines changed: the demo expiry switch (codec.h:14) off; the
#     Linux assembly switch (codec.h:36, 32-bit AT&T inline assembly) off, which selects the
#     reference's portable C++ Tier-1 and DWT; PointerValue (codec.h:197) pointer-sized,
#     since buffers are aligned through it.  "-I-" stops each source from finding the
#     original next to itself, so every file sees the shadow.
#   * <sys/sysctl.h>, gone from glibc, is an empty header in the shim directory, and
#     <cuda_runtime.h> supplies only the integer stream handle of CUDA 1.0, the one CUDA
#     name the GPU manager's headers use (cudainterfacedatatype.h:13-14).
#   * the GPU kernels (gpufunc.cu: legacy texture references) are replaced by
#     oracle/ref_gpu_stub.c, which reports "no GPU"; the engine is run with mUsingGpu false.
#   * the templates that decoderconcrete.cpp uses from bmi_cpu_dwt_decoder.cpp are
#     instantiated by oracle/ref_cpu_dwt_unit.cpp, which compiles that file by #include.
#   * the driver's operator new zero-fills (an uninitialised job-queue member otherwise hangs
#     the engine at random on Linux; see oracle/ref_cpu_driver.cpp).
set -e
REF=${1:-$J2K_REFERENCE_DIR}
[ -n "$REF" ] || { echo "usage: $0 <reference root> (or set J2K_REFERENCE_DIR)" >&2; exit 2; }
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
D="$REF/decoder"
[ -f "$D/codec/include/codec.h" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
SHIM="$OUT/shim"
OBJ="$OUT/obj_cpu"
mkdir -p "$SHIM/sys" "$OBJ"
: > "$SHIM/sys/sysctl.h"
# The GPU manager's headers need only the stream type from the CUDA runtime, and the manager
# compares stream ids with 0, as CUDA 1.0's integer stream handles allowed.
echo 'typedef int cudaStream_t;' > "$SHIM/cuda_runtime.h"
sed -e 's/^#define DEMO_EXPIRE_DATE[[:space:]]*1/#define DEMO_EXPIRE_DATE 0/' \
    -e 's/^\([[:space:]]*#define[[:space:]]*ENABLE_ASSEMBLY_OPTIMIZATION[[:space:]]*\)1/\10/' \
    -e 's/^typedef[[:space:]]*unsigned int[[:space:]]*PointerValue;/typedef unsigned long PointerValue;/' \
    "$D/codec/include/codec.h" > "$SHIM/codec.h"
grep -q '^#define DEMO_EXPIRE_DATE 0' "$SHIM/codec.h" || { echo "codec.h: expiry switch not found" >&2; exit 1; }
grep -q '^typedef unsigned long PointerValue;' "$SHIM/codec.h" || { echo "codec.h: PointerValue not found" >&2; exit 1; }
if grep -q 'ENABLE_ASSEMBLY_OPTIMIZATION[[:space:]]*1' "$SHIM/codec.h"; then
  echo "codec.h: assembly switch still on" >&2; exit 1
fi
INC="-I- -I$SHIM -I$D/codec/include -I$D/codec/src -I$D/common/include -I$D/tools/include -I$D/tools/src \
     -I$D/core/include -I$D/cudainterface/include -I$D/cudainterface/src"
DEFS="-DLINUX -DNDEBUG -D_FINAL"
CXX="g++ -x c++ -std=gnu++98 -fpermissive -w -O2 -fPIC $DEFS"
SRCS=""
for f in dec_init dec_io dec_jp2 dec_packet dec_syntax dec_t1_comp dec_tagtree dec_tsk dec_mq dec_t1_pass dec_dwt \
         bmi_block_decoder bmi_mq_decoder; do
  SRCS="$SRCS $D/codec/src/$f.cpp"
done
SRCS="$SRCS $D/core/src/decoderconcrete.cpp $D/core/src/jobqueue.cpp $D/common/src/decoder.cpp \
      $D/common/src/linuxsemaphore.cpp $D/tools/src/testclock.cpp $D/tools/src/debugtools.cpp \
      $D/core/src/encoderconcrete.cpp $D/cudainterface/src/cudainterface.cpp $D/cudainterface/src/gpulib.c \
      $HERE/ref_cpu_dwt_unit.cpp $HERE/ref_gpu_stub.c $HERE/ref_cpu_driver.cpp"
OBJS=""
for s in $SRCS; do
  o="$OBJ/$(basename "$s").o"
  $CXX $INC -c "$s" -o "$o" 2> "$o.log" || { grep -v "obsolete option" "$o.log" >&2; echo "failed: $s" >&2; exit 1; }
  OBJS="$OBJS $o"
done
g++ -shared -Wl,-Bsymbolic -o "$OUT/libref_cpu.so" $OBJS -lpthread
rm -rf "$OBJ"
echo "built $OUT/libref_cpu.so"
