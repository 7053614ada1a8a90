"""Build recipe of the product library dopamine_b200/_lib/libdopamine_b200.so.

nvcc compiles the CUDA translation units for sm_100a only (-gencode arch=compute_100a,code=sm_100a)
together with the host set-up sources; the library is built in-tree so that it travels with the
working tree.  Usage: python -m dopamine_b200.build [--force]
"""
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libdopamine_b200.so")
CU_SOURCES = ["csrc/cuda/solver.cu", "csrc/cuda/fvm_petsc.cu", "csrc/cuda/noalloc.cu", "csrc/cuda/setup_gpu.cu"]
# The device set-up reproduces the host builder's rounding: no contraction into fused multiply-adds.
CU_FLAGS = {"csrc/cuda/setup_gpu.cu": ["-fmad=false"]}
CPP_SOURCES = ["csrc/host/mesh.cpp", "csrc/host/ops.cpp", "csrc/host/twolevel.cpp", "csrc/host/multilevel.cpp",
               "csrc/host/gmsh.cpp", "csrc/host/foam.cpp"]
HEADERS = ["csrc/cuda/common.cuh", "csrc/cuda/kernels.cuh", "csrc/cuda/pcg.cuh", "csrc/cuda/fcg.cuh",
           "csrc/cuda/learn.cuh", "csrc/cuda/scalars.cuh", "csrc/cuda/mlcg.cuh", "csrc/cuda/mlsolve.cuh", "csrc/cuda/mlkern.cuh", "csrc/cuda/explicit32.cuh",
           "csrc/cuda/setup_gpu.hpp", "csrc/cuda/cellproj.cuh", "csrc/cuda/sampling.cuh", "csrc/cuda/forcing.cuh", "csrc/cuda/sem.cuh", "csrc/host/fortran_records.hpp",
           "csrc/host/twolevel.hpp", "csrc/host/multilevel.hpp", "csrc/host/mesh.hpp", "csrc/host/gmsh.hpp",
           "csrc/host/ops.hpp", "../include/dopamine_b200.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _digest():
    h = hashlib.sha256()
    for rel in CU_SOURCES + CPP_SOURCES + HEADERS + ["build.py"]:
        with open(os.path.join(HERE, rel), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    stamp = os.path.join(OUT_DIR, "build.sha256")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read().strip() == dig:
        return LIB
    nvcc = _nvcc()
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", _host_cxx(), "-I", os.path.join(ROOT, "include")]
    for rel in CU_SOURCES:
        obj = os.path.join(OUT_DIR, os.path.basename(rel) + ".o")
        cmd = [nvcc, *ARCH, "-lineinfo", *common, *CU_FLAGS.get(rel, []), "-Xptxas", "-v" if verbose else "-O3", "-c",
               os.path.join(HERE, rel), "-o", obj]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    for rel in CPP_SOURCES:
        obj = os.path.join(OUT_DIR, os.path.basename(rel) + ".o")
        cmd = [_host_cxx(), "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-c", os.path.join(HERE, rel), "-o", obj]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-ccbin", _host_cxx(), "-Xcompiler", "-fopenmp", "-o", tmp, *objs,
                    "-lcudart"], check=True)
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
