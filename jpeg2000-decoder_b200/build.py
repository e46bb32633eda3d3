"""Build recipe for the native libraries (in-tree, so they travel with the repository).

libj2k_b200.so  host front end (Tier-2), BMI decoder API and the sm_100a kernels
libj2kenc.so    the test/benchmark codestream writer
oracle/liboracle.so, and with a reference tree oracle/_ref/libref_t1.so (its Tier-1) and
oracle/_ref/libref_cpu.so (its whole CPU decoder), are built by `build_oracle`: test and
baseline infrastructure, never linked by the product.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB = os.path.join(PKG, "libj2k_b200.so")
ENC = os.path.join(PKG, "libj2kenc.so")
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF_T1 = os.path.join(ROOT, "oracle", "_ref", "libref_t1.so")
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")

CU_SOURCES = ["engine.cu", "noalloc.cu"]
CPP_SOURCES = ["codestream.cpp", "plan_api.cpp", "bmi_decoder.cpp", "bmi_jp2dec.cpp", "server.cpp"]
HEADERS = ["plan.h", "codestream.h", "t1_kernel.cuh", "t1_lanes.cuh", "dwt_kernel.cuh", "bmi_engine.h",
           "pinned_arena.h"]


def _nvcc():
    for p in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def build_library(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    inc = os.path.join(ROOT, "include")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))]
    hdrs += [os.path.join(inc, h) for h in os.listdir(inc)]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            out = _run([_nvcc()] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
                                           "-I", CSRC, "-I", inc, "-c", s, "-o", o])
            if verbose:
                print(out)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I", CSRC, "-I", inc,
                  "-I", "/usr/local/cuda/include", "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    enc_src = os.path.join(CSRC, "encoder", "j2k_encoder.cpp")
    if force or _stale(ENC, [enc_src, os.path.join(CSRC, "encoder", "j2k_encoder.h")]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", ENC, enc_src, "-lpthread"])
    return LIB


def build_oracle(force=False, reference=None):
    """CPU restatement (always); the reference's Tier-1 and whole CPU decoder when a
    reference tree is given (argument, or the J2K_REFERENCE_DIR environment variable)."""
    src = os.path.join(ROOT, "oracle", "j2k_oracle.c")
    if force or _stale(ORACLE, [src, os.path.join(ROOT, "oracle", "j2k_oracle.h")]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", ORACLE, src])
    reference = reference or os.environ.get("J2K_REFERENCE_DIR")
    if reference and os.path.isdir(os.path.join(reference, "decoder")):
        odir = os.path.join(ROOT, "oracle")
        drv = os.path.join(odir, "ref_t1_driver.cpp")
        if force or _stale(REF_T1, [drv, os.path.join(odir, "build_ref.sh")]):
            _run(["sh", os.path.join(odir, "build_ref.sh"), reference])
        deps = [os.path.join(odir, f) for f in ("build_ref_cpu.sh", "ref_cpu_driver.cpp", "ref_cpu_dwt_unit.cpp",
                                                "ref_gpu_stub.c")]
        if force or _stale(REF_CPU, deps):
            _run(["sh", os.path.join(odir, "build_ref_cpu.sh"), reference])
    return ORACLE


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_oracle(force="--force" in sys.argv)
    print("ok")
