"""Builds the sm_100a library (lib/librlmb.so) and the rlm/hlm command-line drivers (bin/).

    python random-landau-model_b200/build.py [--force]

CUDA sources are compiled by nvcc for sm_100a only; the bit-exact host tables are compiled
by g++ with floating-point contraction off.  Objects go to _build/, outputs stay in-tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "librlmb.so")
BIN = os.path.join(HERE, "bin")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + INCLUDE]

CU_SOURCES = ["heev.cu", "model_kernels.cu", "capi.cu", "profile.cu", "heev_noalloc.cu", "diag_wrappers.cu", "disorder.cu"]
DRIVERS = {"rlm": "tools/rlm_main.cpp", "hlm": "tools/hlm_main.cpp", "rlm_fss": "tools/rlm_fss_main.cpp"}
CPP_SOURCES = ["host_tables.cpp"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "rlm_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            _run([NVCC] + NVFLAGS + ["-c", s, "-o", o])
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            _run([CXX] + CXXFLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    os.makedirs(BIN, exist_ok=True)
    for name, src in DRIVERS.items():
        s = os.path.join(CSRC, src)
        exe = os.path.join(BIN, name)
        deps = [s, LIB, os.path.join(CSRC, "tools", "driver_common.h")]
        if force or _stale(exe, deps):
            _run([CXX, "-O2", "-std=c++17", "-I" + INCLUDE, s, "-o", exe, "-L" + os.path.dirname(LIB),
                  "-lrlmb", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
