"""Build the native library in-tree: dpmmsubclusters_gpu_b200/libdpmm_b200.so.

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
the C++ host driver with g++ and OpenMP.  Objects go to ``_build/`` next to this file;
rebuilds are incremental (an object is rebuilt when any source or header is newer).

    python -m dpmmsubclusters_gpu_b200.build          # or build() from Python
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdpmm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "--expt-relaxed-constexpr",
              "-I" + CSRC, "-I" + INCLUDE] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unknown-pragmas",
             "-I" + CSRC, "-I" + INCLUDE, "-I" + os.path.join(CUDA, "include")]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    return cu, cpp


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(obj: str, src: str, hdr_mtime: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < hdr_mtime


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA / C++ source of the library and link it.  Returns the .so path."""
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = _sources()
    hdr_m = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    jobs = []
    objs = []
    for s in cu:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, s, hdr_m) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", s, "-o", o])
    for s in cpp:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, s, hdr_m):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for err in ex.map(_compile, jobs):
                if verbose and err:
                    sys.stderr.write(err)
    if jobs or not os.path.exists(LIB):
        link = ["g++", "-shared", "-fopenmp", "-o", LIB] + objs + [
            "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
        _compile(link)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
