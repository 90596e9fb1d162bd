"""Builds libngw_b200.so in-tree with nvcc for sm_100a.

    python -m nanogw_b200.build          # or __graft_entry__.build()

CUDA sources get ``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``;
the bit-exact host setup (CVT, Shell sort) is compiled with
``-ffp-contract=off`` so FP64 expressions round where the reference rounds.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libngw_b200.so")
BUILD = os.path.join(HERE, "_build")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels_core.cu", "gemm_tc.cu", "dgemm.cu", "lu.cu", "deflate.cu", "abi.cu", "poisson.cu", "noalloc.cu", "isdf_fit.cu",
              "exchange.cu", "cvt_device.cu", "fft3d.cu"]
CXX_SOURCES = ["host_setup.cpp", "parsec_io.cpp"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "ngw_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xptxas", "-v" if os.environ.get("NGW_PTXAS_V") else "-O3",
                  "-c", s, "-o", o], verbose)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                  "-I", os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o], verbose)
    if force or _stale(OUT, objs):
        tmp = OUT + ".tmp"
        _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcublas", "-lcufft", "-lcusolver", "-lcudart",
              "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")], verbose)
        shutil.move(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
