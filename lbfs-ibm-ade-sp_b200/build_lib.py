"""Builds the in-tree shared library lbfs_b200/_lib/liblbfs_b200.so for sm_100a.

nvcc compiles the CUDA sources for sm_100a only (-gencode
arch=compute_100a,code=sm_100a); the host set-up code is compiled with
-ffp-contract=off so its geometry is bit-identical to the reference's host
code.  Usage: python lbfs-ibm-ade-sp_b200/build_lib.py [--force]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lbfs_b200", "_lib")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liblbfs_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_SOURCES = ["lbfs_fluid.cu", "lbfs_membrane.cu", "lbfs_runtime.cu", "lbfs_noalloc.cu", "lbfs_adjoint.cu", "lbfs_adjoint_mem.cu",
                "lbfs_mesh_gpu.cu"]
HOST_SOURCES = ["host_setup.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _newest_input():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths.append(os.path.join(ROOT, "include", "lbfs_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for src in CUDA_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        jobs.append(([NVCC, *GENCODE, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", *COMMON, "-c",
                      os.path.join(CSRC, src), "-o", obj], obj))
    for src in HOST_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        jobs.append((["g++", "-O2", "-ffp-contract=off", "-fPIC", *COMMON, "-I/usr/local/cuda/include", "-c",
                      os.path.join(CSRC, src), "-o", obj], obj))
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        logs = list(ex.map(lambda j: _run(j[0]), jobs))
    if verbose:
        for log in logs:
            sys.stdout.write(log)
    objs = [j[1] for j in jobs]
    _run([NVCC, *GENCODE, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
