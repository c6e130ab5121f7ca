"""Figures the benchmark's roofline uses, with where each one comes from.

The GEMM main kernel is integer code bound by instruction issue: each SM sub-partition
(4 per SM, 148 SMs on B200) issues at most one warp instruction per cycle.  The roofline
therefore compares the kernel's issued integer-pipe warp instructions per second with
148 * 4 * f_SM warp instructions per second, f_SM being the SM clock sampled during the
run.  The instruction count per posit multiply-add is a property of the compiled kernel
(its fast path is branch-free), measured with ncu on the same kernel and recorded here.
"""

SM_COUNT = 148
SMSP_PER_SM = 4
SM_MAX_MHZ = 1965.0

# Warp instructions issued by gemm_main_kernel per posit multiply-add:
# smsp__inst_executed.sum / (m*n*k) for one NN launch at m = n = k = 4096
# (119,155,165,229 / 68,719,476,736).  Practically all of them are integer ALU or
# integer multiply-add (FMA-pipe) instructions (ALU pipe 61.1 %, FMA pipes 35.0 % busy in
# the same capture; table and operand loads are 0.07 per MAD).
INT_PIPE_WARP_INST_PER_MAD = 1.7339
INST_SOURCE = ("ncu --set full, gemm_main_kernel<false>, NN 4096^3 U[-1,1] "
               "(profiles/gemm_main_kernel_nn_4096.md)")
# DRAM bytes (read + write) per posit multiply-add of the same launch:
# (7,432,703,000 + 73,915,648) / 68,719,476,736.
MAIN_KERNEL_DRAM_BYTES_PER_MAD = 0.1092


def issue_peak_warp_inst_per_s(sm_mhz):
    return SM_COUNT * SMSP_PER_SM * float(sm_mhz) * 1e6
