"""Build the posit32 CUDA library in-tree: ``posit_gpu_b200/libposit_gpu_b200.so``.

nvcc for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``), CUDA runtime
linked statically so the library does not depend on which libcudart the host process
(e.g. torch) already loaded.  Usage: ``python posit_gpu_b200/build.py [-v]``.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libposit_gpu_b200.so")
SOURCES = ["gemm.cu", "lapack.cu", "batch.cu", "batch_gemm.cu", "capi.cu", "batch_capi.cu", "noalloc.cu", "serve.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(HERE, "..", "include", "posit_gpu.h"), os.path.abspath(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.splitext(os.path.basename(s))[0] + ".o")
        cmd = [NVCC] + ARCH + CFLAGS + ["-c", s, "-o", o]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(o)
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
