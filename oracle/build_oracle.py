"""Build recipe for the oracle (test infrastructure).

* ``oracle/liborc.so``        -- the CPU restatement, ``posit_oracle.c`` (always).
* ``oracle/_ref/libposit_ref.so`` -- the reference's OWN sources compiled out of tree
  (only where the reference tree is present): ``libRpack/kernel_entry.cl`` (its
  p32_add / p32_mul, via ``ref_shim/ref_kernel_entry.cpp``) and the untouched
  libRpack CPU BLAS/LAPACK routines, built against ``ref_shim/softposit_cpp.h``.
  Nothing is copied out of the reference tree; outputs go to ``oracle/_ref/`` only.

Usage: ``python oracle/build_oracle.py [--reference DIR]``.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference tree: $POSIT_REFERENCE_DIR, else a directory named "reference" beside this
# repository's root.
REF_DEFAULT = os.environ.get("POSIT_REFERENCE_DIR") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
# The reference CPU routines on the GEMM / LU / Cholesky path (libRpack/Makefile:15-21
# minus the OpenCL glue, iMlaenv (replaced) and util.cpp (LAPACK generators)).
REF_SOURCES = [
    "Rgemm.cpp", "Rsyrk.cpp", "Rtrsm.cpp", "Rgemv.cpp", "Rscal.cpp", "iRamax.cpp",
    "Rlaswp.cpp", "Rgetrf.cpp", "Rgetrf2.cpp", "Rgetrs.cpp", "Rpotrf.cpp", "Rpotrf2.cpp",
    "Rpotrs.cpp", "Mlsame.cpp", "Mxerbla.cpp", "Risnan.cpp",
]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_oracle():
    src = os.path.join(HERE, "posit_oracle.c")
    out = os.path.join(HERE, "liborc.so")
    deps = [src, os.path.join(HERE, "posit_oracle.h")]
    if not _newer(out, deps):
        _run(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-fPIC", "-shared", "-Wall",
              "-o", out, src, "-lm"])
    return out


def build_ref(reference=REF_DEFAULT):
    lib = os.path.join(reference, "libRpack")
    if not os.path.isfile(os.path.join(lib, "kernel_entry.cl")):
        print(f"reference tree not found at {reference}: oracle/_ref not rebuilt", flush=True)
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    out = os.path.join(outdir, "libposit_ref.so")
    shim = os.path.join(HERE, "ref_shim")
    srcs = [os.path.join(lib, s) for s in REF_SOURCES]
    glue = [os.path.join(shim, "ref_kernel_entry.cpp"), os.path.join(shim, "ref_glue.cpp")]
    deps = srcs + glue + [os.path.join(shim, "softposit_cpp.h"), os.path.join(HERE, "posit_oracle.c")]
    if _newer(out, deps):
        return out
    objs = []
    flags = ["-O2", "-fopenmp", "-fPIC", "-std=gnu++17", "-fpermissive", "-w",
             "-D___MPLAPACK_BUILD_WITH__POSIT__", "-I", shim, "-I", lib]
    for s in srcs + glue:
        o = os.path.join(outdir, os.path.splitext(os.path.basename(s))[0] + ".o")
        _run(["g++"] + flags + ["-c", s, "-o", o])
        objs.append(o)
    o = os.path.join(outdir, "posit_oracle.o")
    _run(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-fPIC", "-c",
          os.path.join(HERE, "posit_oracle.c"), "-o", o])
    objs.append(o)
    _run(["g++", "-shared", "-fopenmp", "-o", out] + objs + ["-lm"])
    for o in objs:
        os.remove(o)
    return out


# The reference's GPU-accelerated factorization drivers (they call RgemmG).
REF_DROPIN_SOURCES = ["Rgetrf_opencl.cpp", "Rgetrf2_opencl.cpp", "Rpotrf_opencl.cpp"]


def build_ref_dropin(reference=REF_DEFAULT):
    """oracle/_ref/libposit_ref_dropin.so: the reference CPU routines plus its own
    Rgetrf_opencl / Rgetrf2_opencl / Rpotrf_opencl, unchanged, with RgemmG supplied by
    posit_gpu_b200/integration/Rgemm_b200.cpp over libposit_gpu_b200.so."""
    lib = os.path.join(reference, "libRpack")
    if not os.path.isfile(os.path.join(lib, "Rgetrf_opencl.cpp")):
        print(f"reference tree not found at {reference}: drop-in library not rebuilt", flush=True)
        return None
    root = os.path.dirname(HERE)
    gpu_dir = os.path.join(root, "posit_gpu_b200")
    if not os.path.exists(os.path.join(gpu_dir, "libposit_gpu_b200.so")):
        print("libposit_gpu_b200.so not built: drop-in library not built", flush=True)
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    out = os.path.join(outdir, "libposit_ref_dropin.so")
    shim = os.path.join(HERE, "ref_shim")
    srcs = [os.path.join(lib, s) for s in REF_SOURCES + REF_DROPIN_SOURCES]
    glue = [os.path.join(shim, "ref_kernel_entry.cpp"), os.path.join(shim, "ref_glue.cpp"),
            os.path.join(shim, "ref_dropin_glue.cpp"),
            os.path.join(gpu_dir, "integration", "Rgemm_b200.cpp")]
    deps = srcs + glue + [os.path.join(shim, "softposit_cpp.h"), os.path.join(HERE, "posit_oracle.c"),
                          os.path.join(gpu_dir, "libposit_gpu_b200.so")]
    if _newer(out, deps):
        return out
    objs = []
    flags = ["-O2", "-fopenmp", "-fPIC", "-std=gnu++17", "-fpermissive", "-w",
             "-D___MPLAPACK_BUILD_WITH__POSIT__", "-I", shim, "-I", lib,
             "-I", os.path.join(root, "include")]
    for s in srcs + glue:
        o = os.path.join(outdir, "d_" + os.path.splitext(os.path.basename(s))[0] + ".o")
        _run(["g++"] + flags + ["-c", s, "-o", o])
        objs.append(o)
    o = os.path.join(outdir, "d_posit_oracle.o")
    _run(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-fPIC", "-c",
          os.path.join(HERE, "posit_oracle.c"), "-o", o])
    objs.append(o)
    _run(["g++", "-shared", "-fopenmp", "-o", out] + objs +
         ["-L" + gpu_dir, "-lposit_gpu_b200", "-Wl,-rpath,$ORIGIN/../../posit_gpu_b200", "-lm"])
    for o in objs:
        os.remove(o)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REF_DEFAULT)
    args = ap.parse_args()
    build_oracle()
    build_ref(args.reference)
    build_ref_dropin(args.reference)


if __name__ == "__main__":
    sys.exit(main())
