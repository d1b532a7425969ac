"""Build libvbt_b200.so in-tree: every CUDA source compiled for sm_100a only.

    python vbt_b200/build.py

Device code is compiled with --fmad=false as a safety net (the decode arithmetic already uses
explicitly rounded _rn intrinsics), IEEE division and square root, and -lineinfo for ncu.
Host code is compiled with -ffp-contract=off so host-built weight tables round like the
reference's CPU code.  The CUDA runtime is linked statically.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvbt_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", os.path.join(ROOT, "include"),
              "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
             "-I", "/usr/local/cuda/include"]
CU_SOURCES = ["kernels.cu", "scalar.cu", "capi.cu", "noalloc.cu", "serve.cu", "tune.cu", "sample.cu", "writer.cu", "keyframes.cu"]
CXX_SOURCES = ["facade.cpp"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, ptxas_verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
                if f.endswith(".h")]
    if os.path.isdir(os.path.join(ROOT, "include", "vbt")):
        headers += [os.path.join(ROOT, "include", "vbt", f) for f in os.listdir(os.path.join(ROOT, "include", "vbt"))]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s, __file__] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([NVCC] + ARCH + NVCC_FLAGS + extra + ["-c", s, "-o", o], verbose)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s, __file__] + headers):
            _run(["/usr/bin/g++"] + CXX_FLAGS + ["-c", s, "-o", o], verbose)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
