"""Build recipe for libqumasun_b200.so (sm_100a), in-tree.

    python qumasun-workshop-template_b200/build_lib.py

compiles every csrc/*.cu with nvcc for sm_100a only (csrc/*.cpp, host-only
code, with the host compiler) and links one shared
library next to this file.  The library exports exactly the C ABI declared in
include/qumasun_b200.h.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqumasun_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


CXX = os.environ.get("CXX", "g++")
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-pthread", "-I", os.path.join(ROOT, "include")]


def sources():
    """csrc/*.cu (device code, nvcc) and csrc/*.cpp (host-only code, the host compiler)."""
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "qumasun_b200.h"))
    hdr_mtime = max(os.path.getmtime(h) for h in headers)
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime)):
            continue
        if src.endswith(".cpp"):
            cmd = [CXX] + CXXFLAGS + ["-c", src, "-o", obj]
        else:
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L/usr/local/cuda/lib64", "-lcublas", "-lcusolver", "-lcufft",
            "-Xlinker", "-rpath,/usr/local/cuda/lib64", "-Xcompiler", "-pthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
