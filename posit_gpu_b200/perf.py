"""Figures the benchmark's roofline uses, with where each one comes from.

The GEMM main kernel runs each posit multiply-add as FP64 operations plus a little
integer work (posit32.cuh, f64_posit_mac): it is bound by instruction issue -- each SM
sub-partition (4 per SM, 148 SMs on B200) issues at most one warp instruction per cycle --
with the FP64 pipe (half rate) the busiest pipe.  The roofline therefore compares the
kernel's issued warp instructions per second with 148 * 4 * f_SM warp instructions per
second, f_SM being the SM clock sampled during the run.  The instruction count per posit
multiply-add is a property of the compiled kernel (its fast path is branch-free),
measured with ncu on the same kernel and recorded here.
"""

import hashlib
import os

SM_COUNT = 148
SMSP_PER_SM = 4
SM_MAX_MHZ = 1965.0

# Warp instructions issued by gemm_main_kernel per posit multiply-add:
# smsp__inst_executed.sum / (m*n*k) for one NN launch at m = n = k = 4096
# (48,162,455,398 / 68,719,476,736 = 0.7009, i.e. 22.43 thread instructions).  Of those,
# 10 per multiply-add run on the FP64 pipe (DMUL, DFMA, 6 DADD, 2 DSETP): FP64 pipe
# 62.9 %, ALU pipe 36.1 %, LSU 30.8 %, issue 70.9 % busy in the same capture.
WARP_INST_PER_MAD = 0.7009
FP64_WARP_INST_PER_MAD = 10 / 32
INST_SOURCE = ("ncu --set full, gemm_main_kernel<0,0>, NN 4096^3 U[-1,1] "
               "(profiles/gemm_main_kernel_nn_4096.md)")
# DRAM bytes (read + write) per posit multiply-add of the same launch:
# (7,488,873,000 + 121,976,832) / 68,719,476,736.
MAIN_KERNEL_DRAM_BYTES_PER_MAD = 0.1108


def issue_peak_warp_inst_per_s(sm_mhz):
    return SM_COUNT * SMSP_PER_SM * float(sm_mhz) * 1e6


def fp64_pipe_peak_warp_inst_per_s(sm_mhz):
    """FP64 pipe: 16 lanes per SM sub-partition per cycle, i.e. half a warp instruction."""
    return SM_COUNT * SMSP_PER_SM * 0.5 * float(sm_mhz) * 1e6


# The instruction count above belongs to one build of the main kernel.  It is tied to
# that build by a SHA-256 over the sources that define the kernel's instruction stream
# (gemm.cu and the headers it includes) and the compiler flags (build.py's ARCH and CFLAGS);
# the benchmark recomputes the digest and, when it differs, marks the count stale and
# reports no roofline fraction from it.
KERNEL_SOURCES = ["csrc/gemm.cu", "csrc/gemm.cuh", "csrc/gemm_tile.cuh", "csrc/posit32.cuh"]
INST_SOURCE_DIGEST = "5a203b78e19bc143f412235179eae4c1e55abcb0a85c594a21c4e0e78f9bed8d"


def kernel_source_digest():
    from . import build as _build
    here = os.path.dirname(os.path.abspath(__file__))
    h = hashlib.sha256()
    for rel in KERNEL_SOURCES:
        with open(os.path.join(here, rel), "rb") as fh:
            h.update(rel.encode() + b"\0" + fh.read() + b"\0")
    h.update(b"flags\0" + " ".join(_build.ARCH + _build.CFLAGS).encode() + b"\0")
    return h.hexdigest()


def inst_count_current():
    """True when WARP_INST_PER_MAD was measured on the kernel sources present now."""
    return INST_SOURCE_DIGEST is not None and kernel_source_digest() == INST_SOURCE_DIGEST


# DRAM bytes (read + write) of one main-kernel launch at the LU trailing-update shapes
# m = n = 8192 - b, k = b (key b), from ncu dram__bytes_read.sum + dram__bytes_write.sum
# of that launch.  Empty until measured; the benchmark then reports no traffic figure for
# the shape rather than one scaled from another shape.
TRAILING_TRAFFIC_BYTES = {16: 486810624, 32: 486020096, 64: 487125504, 128: 486207744, 256: 488396800}
TRAILING_TRAFFIC_SOURCE = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum, gemm_main_kernel<0,0>, "
                           "one launch per shape (profiles/gemm_main_kernel_lu_trailing.md)")


def trailing_traffic(k):
    return TRAILING_TRAFFIC_BYTES.get(int(k))
