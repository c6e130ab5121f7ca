#!/usr/bin/env python
"""bench.py -- posit32 Rgemm throughput on B200 (bit-exact, all integer arithmetic).

Workload (one "step"): C <- alpha*op(A)*op(B) + beta*C, posit32, m = n = k = 8192,
transa = transb = 'N', alpha = -1, beta = 1, entries uniform in [-1, 1] (seeded FP64,
converted on the device), column-major, lda = ldb = ldc = 8192 -- the 8192^3 member of
the "posit32 Rgemm at scale" configuration, whose order (beta*C, then c += (alpha*b)*a
over l) is the LU trailing update's.  Metric: posit Gop/s = 2*m*n*k / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: device-resident, through the public device entry point (posit_rgemm_dev,
  including its decode pre-pass), CUDA events on the launching stream, K steps bracketed
  by barrier + synchronize, max over ranks.  A, B and C are 256 MB each and the decoded
  workspace 1 GB, all larger than the 126 MB L2, so no flush is needed between steps.
* e2e: the same GEMM through the host entry point (posit_rgemm, the RgemmG replacement)
  from pinned host buffers: H2D of A, B, C and D2H of C inside the timed region.
* roofline: the main kernel against the SM issue roofline (1 warp instruction per
  cycle per SM sub-partition, 4 per SM, 148 SMs, at the SM clock sampled during the run).
  achieved = integer-pipe warp instructions per launch / main-kernel event time, with
  the instructions per posit multiply-add measured by ncu (posit_gpu_b200/perf.py).
* cpu_baseline: the reference's own CPU Rgemm (libRpack/Rgemm.cpp, OpenMP over columns,
  compiled here into oracle/_ref) on a column slice of the same problem, rank 0, N=1.
* --impl reference: that CPU Rgemm alone, all host threads, each step a column slice.
Multi-GPU (torchrun): independent replicas, one full GEMM per rank (scaling "weak"); the
GEMM has no exchange step, so there is no data-path collective.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 8192
METRIC = "posit32 Rgemm Gop/s (2mnk/t), bit-exact vs CPU Rgemm"
UNIT = "Gop/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--trans", default="NN")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def config(args):
    n = args.n
    return {"workload": f"posit32 Rgemm {args.trans} {n}^3, alpha=-1, beta=1, U[-1,1], column-major, ld={n}",
            "m": n, "n": n, "k": n, "transa": args.trans[0], "transb": args.trans[1],
            "alpha": "-1", "beta": "1", "dist": "uniform[-1,1] (seeded FP64 -> posit32)",
            "l2": "inputs larger than L2 (A, B, C 4*n^2 bytes each + 8*(m+n)*k-byte decoded workspace)",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU"}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref: the reference's own Rgemm) -- cpu_baseline / reference arm
# ---------------------------------------------------------------------------
def cpu_reference_sample(A_host, B_host, C_host, n, trans, cols):
    """Time the reference CPU Rgemm on columns [0, cols) of the n^3 problem."""
    import numpy as np
    import oracle  # checker / CPU baseline only

    lib = oracle.ref
    kind = "reference"
    if lib is None:
        kind = "port"
    ta, tb = trans[0], trans[1]
    Bs = np.ascontiguousarray(B_host[: n * cols]) if tb == "N" else B_host
    Cs = np.ascontiguousarray(C_host[: n * cols]).copy()
    t0 = time.perf_counter()
    if lib is not None:
        lib.ref_rgemm(ta.encode(), tb.encode(), n, cols, n, 0xC0000000, A_host, n, Bs,
                      n if tb == "N" else n, 0x40000000, Cs, n)
    else:
        oracle.orc.orc_rgemm(ta.encode(), tb.encode(), n, cols, n, 0xC0000000, A_host, n, Bs, n,
                             0x40000000, Cs, n)
    dt = time.perf_counter() - t0
    return 2.0 * n * n * cols / dt / 1e9, dt, kind, oracle.orc.orc_num_threads()


def reference_arm(args):
    """--impl reference: the reference's own CPU Rgemm on the host cores."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    n = args.n
    rng = np.random.default_rng(1234)
    threads = oracle.orc.orc_num_threads()
    cols = min(n, 2 * threads)
    A = oracle.from_double(rng.uniform(-1.0, 1.0, size=n * n))
    B = oracle.from_double(rng.uniform(-1.0, 1.0, size=n * n if args.trans[1] != "N" else n * cols))
    C = oracle.from_double(rng.uniform(-1.0, 1.0, size=n * cols))
    times = []
    kind = "reference"
    for i in range(args.warmup + args.steps):
        gops, dt, kind, cores = cpu_reference_sample(A, B, C, n, args.trans, cols)
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = 2.0 * n * n * cols * len(times) / tot / 1e9
    sample = f"columns 0..{cols - 1} of C ({cols} of {n}; per-column work is identical), per step"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * tot / len(times), 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "posit32", "data": "synthetic",
            "config": config(args),
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def ours(args):
    import numpy as np
    import torch

    import posit_gpu_b200 as pg
    from posit_gpu_b200 import perf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    pg.init()
    n = args.n
    ta, tb = args.trans[0], args.trans[1]
    alpha, beta = pg.P32_MINUS_ONE, pg.P32_ONE
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)

    def rand_posit(numel):
        x = torch.rand(numel, dtype=torch.float64, device=dev, generator=g) * 2.0 - 1.0
        return pg.from_double_dev(x)

    A = rand_posit(n * n)
    B = rand_posit(n * n)
    C = rand_posit(n * n)
    ws = torch.empty(pg.workspace_size(ta, tb, n, n, n), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        pg.Rgemm_dev(ta, tb, n, n, n, alpha, A, n, B, n, beta, C, n, workspace=ws, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if pg.device_error(True):
        raise RuntimeError("device error flag raised during warm-up")

    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ
                           else local)
    pg.profile_read(reset=True)
    pg.profile_enable(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    pg.profile_enable(False)
    main_ms, main_launches, all_launches = pg.profile_read(reset=True)
    ms = e0.elapsed_time(e1)
    if pg.device_error(True):
        raise RuntimeError("device error flag raised during the timed region")
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ops_per_step = 2.0 * n * n * n
    value = world * ops_per_step * args.steps / (ms_max / 1e3) / 1e9

    # roofline of the main kernel (issue-bound integer code)
    mads = float(n) * n * n
    main_avg_s = (main_ms / max(1, main_launches)) / 1e3
    sm_mhz = clocks.get("sm_mhz") or perf.SM_MAX_MHZ
    peak = perf.issue_peak_warp_inst_per_s(sm_mhz)
    achieved = None
    if perf.INT_PIPE_WARP_INST_PER_MAD and main_avg_s > 0:
        achieved = perf.INT_PIPE_WARP_INST_PER_MAD * mads / main_avg_s
    roofline = {"bound": "int32_issue", "achieved": achieved and round(achieved / 1e12, 4),
                "peak": round(peak / 1e12, 4), "unit": "T warp-inst/s",
                "frac": achieved and round(achieved / peak, 4),
                "traffic": perf.MAIN_KERNEL_DRAM_BYTES_PER_MAD and perf.MAIN_KERNEL_DRAM_BYTES_PER_MAD * mads,
                "kernel": "gemm_main_kernel<false>" if ta in "nN" else "gemm_main_kernel<true>",
                "main_kernel_ms": round(main_avg_s * 1e3, 3),
                "posit_gop_s_main_kernel": round(2 * mads / main_avg_s / 1e9, 2),
                "int_pipe_warp_inst_per_mad": perf.INT_PIPE_WARP_INST_PER_MAD,
                "peak_basis": f"148 SMs x 4 SMSP x 1 warp-inst/clk at {sm_mhz:.0f} MHz (sampled median)",
                "inst_source": perf.INST_SOURCE}

    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "posit32",
            "data": "synthetic", "config": config(args), "roofline": roofline, "clocks": clocks,
            "gpu_launches": int(all_launches)}

    # end to end through the host entry point (RgemmG replacement), pinned host buffers
    if not args.no_e2e:
        hA = A.cpu().pin_memory()
        hB = B.cpu().pin_memory()
        hC = C.cpu().pin_memory()
        nA, nB, nC = hA.numpy(), hB.numpy(), hC.numpy()
        pg.Rgemm(ta, tb, n, n, n, alpha, nA, n, nB, n, beta, nC, n)  # warm
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        esteps = max(1, min(args.steps, 3))
        for _ in range(esteps):
            pg.Rgemm(ta, tb, n, n, n, alpha, nA, n, nB, n, beta, nC, n)
        e2e_s = time.perf_counter() - t0
        te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_s = float(te.item())
        line["e2e"] = {"value": round(world * ops_per_step * esteps / e2e_s / 1e9, 3), "unit": UNIT,
                       "h2d_bytes_per_step": 3 * 4 * n * n, "d2h_bytes_per_step": 4 * n * n,
                       "steps": esteps, "timing": "host wall clock around the synchronous call"}

    # CPU baseline: the reference's own Rgemm on a column slice, rank 0, N = 1 only
    if world == 1 and not args.no_cpu:
        try:
            import oracle
            threads = oracle.orc.orc_num_threads()
            cols = min(n, 4 * threads)
            hA = A.cpu().numpy().view(np.uint32)
            hB = B.cpu().numpy().view(np.uint32)
            hC = C.cpu().numpy().view(np.uint32)
            gops, dt, kind, cores = cpu_reference_sample(hA, hB, hC, n, args.trans, cols)
            line["cpu_baseline"] = {"value": round(gops, 4), "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": f"columns 0..{cols - 1} of C ({cols} of {n}) of the same "
                                              f"problem, {dt:.1f} s"}
        except Exception as exc:  # the CPU baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                    "sample": f"unavailable: {exc}"}

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
