"""Builds libats_b200.so in-tree (sm_100a only).

    python -m libatssim_b200.build

CUDA sources go through nvcc with -gencode arch=compute_100a,code=sm_100a; the
host topology code is compiled by g++ with -ffp-contract=off so that its float
rest state is evaluated term by term. The shared library lands in
libatssim_b200/lib/ and travels with the source tree.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libats_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I/usr/local/cuda/include"]

CU_SOURCES = ["ats_cloth.cu", "ats_learn.cu", "ats_noalloc.cu"]
CXX_SOURCES = ["ats_topology.cpp", "ats_launcher.cpp", "ats_io.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(os.path.dirname(PKG), "include", "ats_cloth.h"))
    headers.append(os.path.join(os.path.dirname(PKG), "include", "ats_launcher.hpp"))
    headers = [h for h in headers if os.path.exists(h)]
    objs = []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers) or ptxas_info:
            flags = NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else [])
            r = _run([NVCC] + flags + ["-c", "-o", obj, path])
            if verbose or ptxas_info:
                sys.stderr.write(r.stdout + r.stderr)
        objs.append(obj)
    for src in CXX_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers):
            _run([CXX] + CXX_FLAGS + ["-c", "-o", obj, path])
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
