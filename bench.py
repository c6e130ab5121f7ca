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
  achieved = warp instructions per launch / main-kernel event time, with the instructions
  per posit multiply-add measured by ncu (posit_gpu_b200/perf.py); the FP64 pipe's share
  of its own peak is reported beside it.
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
    ap.add_argument("--trailing", type=int, default=0,
                    help="gemm: the LU trailing-update shape m = n = N-b, k = b (b = this value, N = --n)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="gemm: skip the sampled bit-exact check")
    ap.add_argument("--workload", default="gemm", choices=["gemm", "lu", "cholesky", "batch", "serve"],
                    help="gemm (default, the headline), lu / cholesky (device-resident "
                         "factorization + solve, FP64 errors), batch (batched vs per-call)")
    ap.add_argument("--nb", type=int, default=0, help="panel width for lu/cholesky (0: tuned)")
    ap.add_argument("--problems", type=int, default=20000, help="batch: factor-and-solve problems")
    ap.add_argument("--gemms", type=int, default=50000, help="batch: GEMM problems")
    ap.add_argument("--requests", type=int, default=300, help="serve: requests per arrival rate")
    ap.add_argument("--rates", default="5,10,20,40,burst", help="serve: Poisson arrival rates (req/s)")
    ap.add_argument("--per-call-sample", type=int, default=0,
                    help="serve: requests timed on the per-call path (0: all of them)")
    ap.add_argument("--batch-max-n", type=int, default=0, help="serve: batched-kernel size limit (0: default)")
    ap.add_argument("--lanes", type=int, default=0, help="serve: CUDA streams of the server (0: default)")
    ap.add_argument("--launch-threads", type=int, default=0, help="serve: launcher threads (0: default)")
    ap.add_argument("--serve-nb", type=int, default=0, help="serve: the server's panel width (0: its default)")
    ap.add_argument("--serve-priority-n", type=int, default=0,
                    help="serve: n from which requests run on high-priority lanes (0: default, -1: none)")
    ap.add_argument("--profile-path", default="", choices=["", "percall", "served"],
                    help="serve: bracket only this path with cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off); both paths still run")
    return ap.parse_args()


def shape(args):
    """(m, n, k) of the GEMM arm: N^3, or the trailing-update shape (N-b) x (N-b) x b."""
    if args.trailing:
        return args.n - args.trailing, args.n - args.trailing, args.trailing
    return args.n, args.n, args.n


def config(args):
    m, n, k = shape(args)
    what = (f"{m}x{n}x{k} (LU trailing update of {args.n}, b={k})" if args.trailing else f"{n}^3")
    l2 = ("inputs larger than L2 (A, B, C 4*n^2 bytes each + 8*(m+n)*k-byte decoded workspace)"
          if not args.trailing else "C (4*m*n bytes) larger than L2")
    return {"workload": f"posit32 Rgemm {args.trans} {what}, alpha=-1, beta=1, U[-1,1], column-major",
            "m": m, "n": n, "k": k, "transa": args.trans[0], "transb": args.trans[1],
            "alpha": "-1", "beta": "1", "dist": "uniform[-1,1] (seeded FP64 -> posit32)", "l2": l2,
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
# multi-rank timing: every rank times its own replica; the job's time is the slowest
# rank's, and the job's rate counts the work of all ranks
# ---------------------------------------------------------------------------
def max_over_ranks(x, dist, device):
    """x, maximised over the ranks of the default process group (dist None: one rank)."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, work_per_step, steps, ms_max):
    """Units per second of the whole job: world replicas, `steps` steps each, in ms_max."""
    return world * work_per_step * steps / (ms_max / 1e3)


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
    m, n, k = shape(args)
    ta, tb = args.trans[0], args.trans[1]
    alpha, beta = pg.P32_MINUS_ONE, pg.P32_ONE
    from posit_gpu_b200 import workloads
    A, lda, B, ldb, C, _ = workloads.gemm_operands(m, n, k, ta, tb, seed=workloads.GEMM_SEED + rank, device=dev)
    ws = torch.empty(pg.workspace_size(ta, tb, m, n, k), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        pg.Rgemm_dev(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, m, workspace=ws, stream=stream)

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
    ms_max = max_over_ranks(ms, dist, dev)
    ops_per_step = 2.0 * m * n * k
    value = whole_job_rate(world, ops_per_step, args.steps, ms_max) / 1e9

    # roofline of the main kernel: instruction issue (FP64 pipe the busiest pipe)
    mads = float(m) * n * k
    main_avg_s = main_ms / 1e3 / max(main_launches, 1) if main_launches else 0.0
    sm_mhz = clocks.get("sm_mhz") or perf.SM_MAX_MHZ
    peak = perf.issue_peak_warp_inst_per_s(sm_mhz)
    achieved = None
    current = perf.inst_count_current()
    if perf.WARP_INST_PER_MAD and main_avg_s > 0 and current:
        achieved = perf.WARP_INST_PER_MAD * mads / main_avg_s
    fp64_frac = (perf.FP64_WARP_INST_PER_MAD * mads / main_avg_s / perf.fp64_pipe_peak_warp_inst_per_s(sm_mhz)
                 if main_avg_s > 0 else None)
    roofline = {"bound": "issue", "achieved": achieved and round(achieved / 1e12, 4),
                "peak": round(peak / 1e12, 4), "unit": "T warp-inst/s",
                "frac": achieved and round(achieved / peak, 4),
                "traffic": (perf.MAIN_KERNEL_DRAM_BYTES_PER_MAD * mads
                            if perf.MAIN_KERNEL_DRAM_BYTES_PER_MAD and not args.trailing else None),
                "kernel": "gemm_main_kernel<false,false>" if ta in "nN" else "gemm_main_kernel<true,false>",
                "main_kernel_ms": round(main_avg_s * 1e3, 3),
                "posit_gop_s_main_kernel": round(2 * mads / main_avg_s / 1e9, 2) if main_avg_s > 0 else None,
                "warp_inst_per_mad": perf.WARP_INST_PER_MAD,
                "fp64_pipe_frac": fp64_frac and round(fp64_frac, 4),
                "peak_basis": f"148 SMs x 4 SMSP x 1 warp-inst/clk at {sm_mhz:.0f} MHz (sampled median); "
                              "MEASURED_PEAKS.json has no issue or FP64 figure",
                "inst_source": perf.INST_SOURCE,
                "inst_source_stale": not current,
                "kernel_source_sha256": perf.kernel_source_digest()}
    if not current:
        roofline["fp64_pipe_frac"] = None
    if args.trailing:  # measured per shape, never scaled from the cube
        roofline["traffic"] = perf.trailing_traffic(k)
        roofline["traffic_source"] = perf.TRAILING_TRAFFIC_SOURCE if roofline["traffic"] else "not measured"

    if args.trailing:
        # short k: HBM reported beside the issue roofline (algorithmic bytes 4*(mk + kn + 2mn))
        alg = 4.0 * (m * k + k * n + 2.0 * m * n)
        step_s = ms_max / args.steps / 1e3
        peak_gbs, basis = None, "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                peak_gbs = json.load(fh).get("hbm_gbs")
        except (OSError, ValueError):
            pass
        if not peak_gbs:  # the file is absent here: the earlier measurement on B200 (copy, 6.65 TB/s)
            peak_gbs, basis = 6650.0, "fallback: 6650 GB/s measured copy bandwidth on B200 (no MEASURED_PEAKS.json)"
        roofline["hbm"] = {"algorithmic_bytes": alg, "achieved_gbs": round(alg / step_s / 1e9, 1),
                           "peak_gbs": peak_gbs, "frac": round(alg / step_s / 1e9 / peak_gbs, 4),
                           "peak_basis": basis}

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
        pg.Rgemm(ta, tb, m, n, k, alpha, nA, lda, nB, ldb, beta, nC, m)  # warm
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        esteps = max(1, min(args.steps, 3))
        for _ in range(esteps):
            pg.Rgemm(ta, tb, m, n, k, alpha, nA, lda, nB, ldb, beta, nC, m)
        e2e_s = time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, dist, dev)
        line["e2e"] = {"value": round(world * ops_per_step * esteps / e2e_s / 1e9, 3), "unit": UNIT,
                       "h2d_bytes_per_step": 4 * (m * k + k * n + m * n), "d2h_bytes_per_step": 4 * m * n,
                       "steps": esteps, "timing": "host wall clock around the synchronous call"}

    # CPU baseline: the reference's own Rgemm on a column slice, rank 0, N = 1 only
    if world == 1 and not args.no_cpu and not args.trailing:
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

    # bit-exact check of the benched kernel on its own problem: one more step on a copy of
    # the current C, sampled columns against the reference's own CPU Rgemm (rank 0)
    if rank == 0 and not args.no_check:
        line["bit_exact_sample"] = bit_exact_sample(pg, A, lda, B, ldb, C, m, n, k, ta, tb, alpha, beta, ws,
                                                    stream)

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bit_exact_sample(pg, A, lda, B, ldb, C, m, n, k, ta, tb, alpha, beta, ws, stream, width=8):
    """One step of the benched GEMM on a copy of C, compared on sampled columns (all
    rows of the first, middle and last `width` columns) with the reference's own CPU Rgemm
    (oracle/_ref; the restatement where that was not built)."""
    import numpy as np
    import torch
    try:
        import oracle  # checker only
        Cout = C.clone()
        pg.Rgemm_dev(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cout, m, workspace=ws, stream=stream)
        torch.cuda.synchronize()
        hA = A.cpu().numpy().view(np.uint32)
        hB = B.cpu().numpy().view(np.uint32)
        hC = C.cpu().numpy().view(np.uint32)
        got = Cout.cpu().numpy().view(np.uint32)
        mid = (n // 2) // width * width
        spans = sorted({(0, min(width, n)), (mid, min(mid + width, n)), (max(0, n - width), n)})
        t0 = time.perf_counter()
        bad, kind = 0, None
        for j0, j1 in spans:
            want, kind = oracle.rgemm_cols_checked(ta, tb, m, n, k, alpha, hA, lda, hB, ldb, beta, hC, m, j0, j1)
            bad += int(np.count_nonzero(got[j0 * m:j1 * m] != want))
        return {"ok": bad == 0, "mismatches": bad, "entries": sum(j1 - j0 for j0, j1 in spans) * m,
                "columns": [[j0, j1 - 1] for j0, j1 in spans], "checker": kind,
                "check_s": round(time.perf_counter() - t0, 1)}
    except Exception as exc:  # reported; a failed check is never hidden
        return {"ok": False, "error": str(exc)}


# ---------------------------------------------------------------------------
# device-resident factorization (configuration 3) and batching (configuration 4)
# ---------------------------------------------------------------------------
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def factor_arm(args):
    """LU or Cholesky of one n x n system, nb from the tuner: posit Gop/s with the
    reference's work formulas ((2/3)n^3 LU, (1/3)n^3 Cholesky; main_lu_bench.cpp:102,
    main_cholesky_bench.cpp:113), the solve, and the FP64 error report."""
    import torch

    import posit_gpu_b200 as pg
    from posit_gpu_b200 import accuracy, autotune
    n = args.n
    lu = args.workload == "lu"
    nb = args.nb or autotune.panel_width(n, "lu" if lu else "chol")
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(4242)
    if lu:
        A0 = pg.from_double_dev(torch.rand(n * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    else:
        M = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        S = M @ M.t() / n + torch.eye(n, dtype=torch.float64, device=dev)
        A0 = pg.from_double_dev(S.t().contiguous().reshape(-1))
        del M, S
    x = pg.from_double_dev(torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    b = torch.zeros(n, dtype=torch.int32, device=dev)
    pg.Rgemm_dev("N", "N", n, 1, n, pg.P32_ONE, A0, n, x, n, 0, b, n)
    A = A0.clone()
    ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def factor():
        if lu:
            pg.Rgetrf_dev(n, n, A, n, ipiv, info, nb=nb)
        else:
            pg.Rpotrf_dev("L", n, A, n, info, nb=nb)

    times = []
    sampler = ClockSampler(torch.cuda.current_device())
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            sampler.start()
        A.copy_(A0)
        e0, e1 = _events()
        e0.record()
        factor()
        e1.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = sum(times) / len(times)
    rhs = b.clone()
    e0, e1 = _events()
    e0.record()
    if lu:
        pg.Rgetrs_dev("N", n, 1, A, n, ipiv, rhs, n)
    else:
        pg.Rpotrs_dev("L", n, 1, A, n, rhs, n)
    e1.record()
    torch.cuda.synchronize()
    solve_ms = e0.elapsed_time(e1)
    work = (2.0 if lu else 1.0) / 3.0 * n ** 3
    rep = accuracy.solve_report(A0, b, rhs, x_true=x, n=n, spd=not lu)
    cpu = None
    if not args.no_cpu:
        # the reference's own CPU Rgetrf / Rpotrf (oracle/_ref), full factorization of the
        # leading block of the same matrix (same distribution), same nb
        try:
            import numpy as np

            import oracle
            nc = min(n, 1024)
            blk = A0.view(n, n).t()[:nc, :nc].t().contiguous().cpu().numpy().view(np.uint32).reshape(-1).copy()
            piv = np.zeros(nc, dtype=np.int32)
            t0 = time.perf_counter()
            if oracle.ref is not None:
                kind = "reference"
                (oracle.ref.ref_rgetrf(nc, nc, blk, nc, piv, nb) if lu else oracle.ref.ref_rpotrf(b"L", nc, blk, nc, nb))
            else:
                kind = "port"
                (oracle.orc.orc_rgetrf(nc, nc, blk, nc, piv, nb) if lu else oracle.orc.orc_rpotrf(b"L", nc, blk, nc, nb))
            dt = time.perf_counter() - t0
            cwork = (2.0 if lu else 1.0) / 3.0 * nc ** 3
            cpu = {"value": round(cwork / dt / 1e9, 4), "unit": "Gop/s", "cores": oracle.orc.orc_num_threads(),
                   "kind": kind, "sample": f"full {'Rgetrf' if lu else 'Rpotrf(L)'} of the leading {nc}x{nc} block "
                                           f"of the same matrix, nb={nb}, {dt:.1f} s"}
        except Exception as exc:  # reported, never required
            cpu = {"value": None, "unit": "Gop/s", "cores": None, "kind": "reference", "sample": f"unavailable: {exc}"}
    line = {"metric": f"posit32 {'Rgetrf' if lu else 'Rpotrf(L)'} Gop/s ({'2/3' if lu else '1/3'} n^3 / t), "
                      f"device-resident, bit-exact vs CPU", "value": round(work / (ms / 1e3) / 1e9, 3),
            "unit": "Gop/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "posit32",
            "data": "synthetic", "config": {"workload": f"{args.workload} n={n} nb={nb}, "
                                                        f"{'U[-1,1]' if lu else 'M*M^T/n + I, M ~ U[-1,1]'}, "
                                                        "one right-hand side b = A*x_true"},
            "info": int(info.item()), "solve_ms": round(solve_ms, 3), "fp64_report": rep, "clocks": clocks}
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def _logu(rng, lo, hi, size):
    import numpy as np
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size))).astype(int)


def batch_arm(args):
    """Configuration 4: 20,000 LU/Cholesky factor-and-solve problems (n log-uniform 8..512)
    and 50,000 GEMMs (m, n, k log-uniform 4..512, random transposes), batched (one
    persistent graph-captured launch each) against the plain per-call path on a sample."""
    import numpy as np
    import torch

    import posit_gpu_b200 as pg
    from posit_gpu_b200 import autotune
    dev = torch.device("cuda")
    rng = np.random.default_rng(20260101)
    g = torch.Generator(device=dev)
    g.manual_seed(99)
    P = args.problems
    ns = _logu(rng, 8, 512, P)
    kinds = np.where(rng.random(P) < 0.5, pg.BATCH_LU, pg.BATCH_CHOLESKY)
    # one arena per kind of buffer
    offA = np.concatenate([[0], np.cumsum(ns * ns)])
    offB = np.concatenate([[0], np.cumsum(ns)])
    A0 = pg.from_double_dev(torch.rand(int(offA[-1]), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    X = pg.from_double_dev(torch.rand(int(offB[-1]), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    for i in np.nonzero(kinds == pg.BATCH_CHOLESKY)[0]:
        n = int(ns[i])
        M = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        S = (M @ M.t() / n + torch.eye(n, dtype=torch.float64, device=dev)).t().contiguous().reshape(-1)
        A0[offA[i]:offA[i + 1]] = pg.from_double_dev(S)
    B0 = torch.zeros_like(X)
    view = lambda t, o, i: t[int(o[i]):int(o[i + 1])]
    rhs_plan = pg.BatchGemmPlan([("N", "N", int(ns[i]), 1, int(ns[i]), pg.P32_ONE, view(A0, offA, i), int(ns[i]),
                                  view(X, offB, i), int(ns[i]), 0, view(B0, offB, i), int(ns[i])) for i in range(P)])
    rhs_plan.launch()  # b = A*x_true for every problem, batched (Rgemv 'N' bits)
    A = A0.clone()
    B = B0.clone()
    ipiv = torch.zeros(int(offB[-1]), dtype=torch.int32, device=dev)
    info = torch.zeros(P, dtype=torch.int32, device=dev)
    plan = pg.BatchPlan([(int(kinds[i]), view(A, offA, i), view(B, offB, i), view(ipiv, offB, i), info[i:i + 1])
                         for i in range(P)])
    times = []
    sampler = ClockSampler(torch.cuda.current_device())
    for r in range(args.warmup + args.steps):
        if r == args.warmup:
            sampler.start()
        A.copy_(A0)
        B.copy_(B0)
        e0, e1 = _events()
        e0.record()
        plan.launch()
        e1.record()
        torch.cuda.synchronize()
        if r >= args.warmup:
            times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    batch_ms = sum(times) / len(times)
    # per-call path on a sample (same problems, same order)
    S_ = min(P, 400)
    Ac = A0.clone()
    Bc = B0.clone()
    ipc = torch.zeros_like(ipiv)
    infc = torch.zeros_like(info)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for i in range(S_):
        n = int(ns[i])
        a, b_, ip = view(Ac, offA, i), view(Bc, offB, i), view(ipc, offB, i)
        if kinds[i] == pg.BATCH_LU:
            pg.Rgetrf_dev(n, n, a, n, ip, infc[i:i + 1])
            pg.Rgetrs_dev("N", n, 1, a, n, ip, b_, n)
        else:
            pg.Rpotrf_dev("L", n, a, n, infc[i:i + 1])
            pg.Rpotrs_dev("L", n, 1, a, n, b_, n)
    e1.record()
    torch.cuda.synchronize()
    percall_ms = e0.elapsed_time(e1)
    same = all(torch.equal(view(Ac, offA, i), view(A, offA, i)) and torch.equal(view(Bc, offB, i), view(B, offB, i))
               for i in range(S_))
    # GEMM batch
    G = args.gemms
    gm, gn, gk = _logu(rng, 4, 512, G), _logu(rng, 4, 512, G), _logu(rng, 4, 512, G)
    ta = rng.choice(["N", "T"], G)
    tb = rng.choice(["N", "T"], G)
    oA = np.concatenate([[0], np.cumsum(gm * gk)])
    oB = np.concatenate([[0], np.cumsum(gk * gn)])
    oC = np.concatenate([[0], np.cumsum(gm * gn)])
    GA = pg.from_double_dev(torch.rand(int(oA[-1]), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    GB = pg.from_double_dev(torch.rand(int(oB[-1]), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    GC0 = pg.from_double_dev(torch.rand(int(oC[-1]), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
    GC = GC0.clone()

    def gprob(i, C):
        m, n, k = int(gm[i]), int(gn[i]), int(gk[i])
        return (ta[i], tb[i], m, n, k, pg.P32_MINUS_ONE, view(GA, oA, i), m if ta[i] == "N" else k,
                view(GB, oB, i), k if tb[i] == "N" else n, pg.P32_ONE, view(C, oC, i), m)

    gplan = pg.BatchGemmPlan([gprob(i, GC) for i in range(G)], tile_table=autotune.gemm_tile_table())
    gt = []
    gsampler = ClockSampler(torch.cuda.current_device())
    for r in range(args.warmup + args.steps):
        if r == args.warmup:
            gsampler.start()
        GC.copy_(GC0)
        e0, e1 = _events()
        e0.record()
        gplan.launch()
        e1.record()
        torch.cuda.synchronize()
        if r >= args.warmup:
            gt.append(e0.elapsed_time(e1))
    gclocks = gsampler.stop()
    gbatch_ms = sum(gt) / len(gt)
    ops = float(np.sum(2.0 * gm * gn * gk))
    GS = min(G, 2000)
    GCc = GC0.clone()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for i in range(GS):
        pg.Rgemm_dev(*gprob(i, GCc))
    e1.record()
    torch.cuda.synchronize()
    gpercall_ms = e0.elapsed_time(e1)
    gsame = all(torch.equal(view(GCc, oC, i), view(GC, oC, i)) for i in range(GS))
    ops_s = float(np.sum(2.0 * gm[:GS] * gn[:GS] * gk[:GS]))
    value = P / (batch_ms / 1e3)
    line = {"metric": "batched posit32 LU/Cholesky factor+solve solves/s (20,000 problems, n log-uniform 8..512)",
            "value": round(value, 1), "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(batch_ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "posit32", "data": "synthetic",
            "config": {"workload": "config 4: 50% LU / 50% Cholesky(L), nrhs 1, b = A*x_true; "
                                   "50,000 GEMMs m,n,k log-uniform 4..512, random transposes, alpha=-1, beta=1"},
            "per_call_solves_per_s": round(S_ / (percall_ms / 1e3), 1), "per_call_sample": S_,
            "speedup_vs_per_call": round(value / (S_ / (percall_ms / 1e3)), 2),
            "bit_identical_to_per_call_on_sample": bool(same),
            "gemm_batch": {"gemms": G, "ms": round(gbatch_ms, 3), "gop_s": round(ops / (gbatch_ms / 1e3) / 1e9, 2),
                           "gemms_per_s": round(G / (gbatch_ms / 1e3), 1),
                           "per_call_gop_s": round(ops_s / (gpercall_ms / 1e3) / 1e9, 2),
                           "per_call_gemms_per_s": round(GS / (gpercall_ms / 1e3), 1), "per_call_sample": GS,
                           "bit_identical_to_per_call_on_sample": bool(gsame),
                           "tile_table": autotune.gemm_tile_table(), "clocks": gclocks},
            "max_info": int(info.max().item()), "clocks": clocks}
    print(json.dumps(line), flush=True)
    return 0


def _serve_workload(R, seed=5150):
    """Configuration 5's request stream: LU / Cholesky 50/50, n log-uniform 32..4096,
    nrhs uniform 1..16, 30% of requests reusing an earlier request's matrix (kind and n
    included) with new right-hand sides.  Returns per-request (kind, n, nrhs, matrix id)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    kinds = np.where(rng.random(R) < 0.5, 0, 1)
    ns = _logu(rng, 32, 4096, R)
    nrhs = rng.integers(1, 17, R)
    mid = np.arange(R)
    for i in range(1, R):
        if rng.random() < 0.3:
            j = int(rng.integers(0, i))
            mid[i], kinds[i], ns[i] = mid[j], kinds[j], ns[j]
    return [(int(kinds[i]), int(ns[i]), int(nrhs[i]), int(mid[i])) for i in range(R)]


def _serve_data(reqs):
    """Matrices (config 3's distributions: U[-1,1] for LU, M*M^T/n + I for Cholesky) seeded
    per matrix, right-hand sides B = A*X_true (FP64 of the posit values, X_true ~ U[-1,1])
    seeded per request; everything lands in page-locked host buffers."""
    import torch

    import posit_gpu_b200 as pg
    dev = torch.device("cuda")
    f64 = torch.float64
    mats, rhs = {}, []
    for i, (kind, n, r, m) in enumerate(reqs):
        g = torch.Generator(device=dev)
        if m not in mats:
            g.manual_seed(1_000_003 * m + 17)
            if kind == 0:
                Ad = pg.from_double_dev(torch.rand(n * n, dtype=f64, device=dev, generator=g) * 2 - 1)
            else:
                M = torch.rand(n, n, dtype=f64, device=dev, generator=g) * 2 - 1
                Ad = pg.from_double_dev((M @ M.t() / n + torch.eye(n, dtype=f64, device=dev)).reshape(-1))
                del M
            host = torch.empty(n * n, dtype=torch.int32, pin_memory=True)
            host.copy_(Ad)
            mats[m] = host
        g.manual_seed(7_000_001 * i + 5)
        A64 = pg.to_double_dev(mats[m].to(dev)).reshape(n, n).t()  # column-major
        X64 = pg.to_double_dev(pg.from_double_dev(torch.rand(n * r, dtype=f64, device=dev, generator=g) * 2 - 1))
        B64 = A64 @ X64.reshape(r, n).t()
        Bh = torch.empty(n * r, dtype=torch.int32, pin_memory=True)
        Bh.copy_(pg.from_double_dev(B64.t().contiguous().reshape(-1)))
        rhs.append(Bh)
    torch.cuda.synchronize()
    return mats, rhs


def _percentile(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs), q)) if len(xs) else None


def serve_arm(args):
    """Configuration 5: served Ax = b requests at Poisson arrival rates (and a burst),
    through the library's request loop (posit_server_*): continuous admission under the
    150 GB device budget, batched small systems, blocked large ones overlapping on the GPU,
    factors cached on the device for repeat matrices.  Against the plain per-call drop-in
    path (posit_rgetrf + posit_rgetrs / posit_rpotrf + posit_rpotrs on host buffers, one
    request after another, reusing host-side factors for repeat matrices) on a sample of
    the same stream.  Every served solution is compared bit for bit with the per-call one
    and across rates.  Times are host wall-clock from submit to the solution in host
    memory (end to end: H2D of A and B, D2H of X inside)."""
    import numpy as np
    import torch

    import posit_gpu_b200 as pg
    R = args.requests
    reqs = _serve_workload(R)
    mats, rhs = _serve_data(reqs)
    zeros = lambda i: torch.zeros(reqs[i][1] * reqs[i][2], dtype=torch.int32, pin_memory=True)

    # plain per-call path, one request after another
    S = min(R, args.per_call_sample) if args.per_call_sample > 0 else R
    fac_src = {m: mats[m].numpy().view(np.uint32).copy() for (_, _, _, m) in reqs[:S]}
    xs = [rhs[i].numpy().view(np.uint32).copy() for i in range(S)]
    pc_info, factors, pc_lat = [], {}, []
    if args.profile_path == "percall":
        torch.cuda.profiler.start()
    t0 = time.perf_counter()
    for i in range(S):
        kind, n, r, m = reqs[i]
        ts = time.perf_counter()
        if m not in factors:
            F = fac_src[m]
            ipiv = np.zeros(n, np.int32)
            info = pg.Rgetrf(n, n, F, n, ipiv) if kind == 0 else pg.Rpotrf("L", n, F, n)
            factors[m] = (F, ipiv, info)
        F, ipiv, info = factors[m]
        if kind == 0:
            pg.Rgetrs("N", n, r, F, n, ipiv, xs[i], n)
        elif info == 0:
            pg.Rpotrs("L", n, r, F, n, xs[i], n)
        pc_info.append(info)
        pc_lat.append((time.perf_counter() - ts) * 1e3)
    pc_s = time.perf_counter() - t0
    if args.profile_path == "percall":
        torch.cuda.profiler.stop()
    pc_rate = S / pc_s

    # served, at each arrival rate
    rates = [r.strip() for r in args.rates.split(",") if r.strip()]
    runs, served_x, clocks = [], None, None
    same_across = True
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    if args.profile_path == "served":
        torch.cuda.profiler.start()
    for rate in rates:
        outs = [zeros(i) for i in range(R)]
        arng = np.random.default_rng(77)
        gaps = np.zeros(R) if rate == "burst" else arng.exponential(1.0 / float(rate), R)
        arrive = np.cumsum(gaps) - gaps[0]
        with pg.Server(batch_max_n=args.batch_max_n, lanes=args.lanes, launch_threads=args.launch_threads,
                       nb=args.serve_nb, priority_n=args.serve_priority_n) as srv:
            tickets, t_sub = [None] * R, [0.0] * R

            def feed():
                base = time.perf_counter()
                for i, (kind, n, r, m) in enumerate(reqs):
                    delay = base + arrive[i] - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    t_sub[i] = time.perf_counter()
                    tickets[i] = srv.submit(kind, n, r, mats[m], rhs[i], outs[i], matrix_id=m)

            th = threading.Thread(target=feed)
            th.start()
            th.join()
            res = [srv.wait(t) for t in tickets]
            st = srv.stats()
        lat = [x["latency_ms"] for x in res]
        span = max(t_sub[i] + lat[i] / 1e3 for i in range(R)) - t_sub[0]
        ok = all(x["status"] == 0 for x in res)
        hits = sum(x["cache_hit"] for x in res)
        xs_run = [o.numpy().view(np.uint32) for o in outs]
        bad_pc = [i for i in range(S)
                  if res[i]["info"] != pc_info[i] or (pc_info[i] == 0 and not np.array_equal(xs_run[i], xs[i]))]
        same_pc = not bad_pc
        mismatches = [{"i": i, "kind": reqs[i][0], "n": reqs[i][1], "nrhs": reqs[i][2], "path": res[i]["path"],
                       "hit": res[i]["cache_hit"], "info": res[i]["info"], "want_info": pc_info[i]}
                      for i in bad_pc[:8]]
        if served_x is None:
            served_x = (xs_run, [x["info"] for x in res])
        else:
            same_across &= all(served_x[1][i] == res[i]["info"] and
                               (res[i]["info"] != 0 or np.array_equal(served_x[0][i], xs_run[i])) for i in range(R))
        by_path = {p: [x["latency_ms"] for x in res if x["path"] == p] for p in (0, 1)}
        slow = sorted(range(R), key=lambda i: -lat[i])[:4]
        slowest = [{"kind": "LU" if reqs[i][0] == 0 else "Cholesky", "n": reqs[i][1], "nrhs": reqs[i][2],
                    "path": res[i]["path"], "hit": res[i]["cache_hit"], "ms": round(lat[i], 1),
                    "queue_ms": round(res[i]["queue_ms"], 1)} for i in slow]
        runs.append({"rate_req_s": rate, "solves_per_s": round(R / span, 2),
                     "rhs_per_s": round(sum(q[2] for q in reqs) / span, 1),
                     "p50_ms": round(_percentile(lat, 50), 2), "p99_ms": round(_percentile(lat, 99), 2),
                     "p50_queue_ms": round(_percentile([x["queue_ms"] for x in res], 50), 3),
                     "p99_batched_ms": round(_percentile(by_path[0], 99) or 0, 2),
                     "p99_blocked_ms": round(_percentile(by_path[1], 99) or 0, 2),
                     "all_ok": ok, "cache_hits": hits, "inflight_peak": st["inflight_peak"],
                     "batched_units": st["batched_units"], "blocked_units": st["blocked_units"],
                     "evictions": st["evictions"], "bytes_peak_gb": round(st["bytes_peak"] / 1e9, 2),
                     "bit_identical_to_per_call_on_sample": bool(same_pc), "mismatches": mismatches,
                     "slowest": slowest})
    if args.profile_path == "served":
        torch.cuda.profiler.stop()
    clocks = sampler.stop()
    repeats = sum(1 for i, q in enumerate(reqs) if q[3] != i)
    best = max(runs, key=lambda x: x["solves_per_s"])
    h2d = sum(4 * (q[1] * q[1] + q[1] * q[2]) for q in reqs) / R
    line = {"metric": "served posit32 Ax=b solves/s (LU/Cholesky, n log-uniform 32..4096, nrhs 1..16), "
                      "p50/p99 latency, bit-identical to per-call",
            "value": best["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": len(rates), "warmup": 0,
            "ms_per_step": round(1e3 / best["solves_per_s"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "posit32", "data": "synthetic",
            "config": {"workload": f"config 5: {R} requests, 50% LU / 50% Cholesky(L), {repeats} repeat "
                                   "matrices (30%), B = A*X_true, Poisson arrivals per rate, 150 GB budget",
                       "rates": rates, "batch_max_n": args.batch_max_n or 256,
                       "server_nb": args.serve_nb or "max(32, tuned) per n",
                       "server_priority_n": args.serve_priority_n or "default (2048)"},
            "e2e": {"value": best["solves_per_s"], "unit": "solves/s", "h2d_bytes_per_step": round(h2d),
                    "d2h_bytes_per_step": round(sum(4 * q[1] * q[2] for q in reqs) / R),
                    "note": "value is itself end to end: host buffers in, solution in host memory"},
            "rates": runs, "per_call": {"solves_per_s": round(pc_rate, 2), "sample": S,
                                        "p50_ms": round(_percentile(pc_lat, 50), 2),
                                        "p99_ms": round(_percentile(pc_lat, 99), 2)},
            "speedup_vs_per_call": round(best["solves_per_s"] / pc_rate, 2),
            "bit_identical_across_rates": bool(same_across), "clocks": clocks}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload in ("lu", "cholesky"):
        return factor_arm(args)
    if args.workload == "batch":
        return batch_arm(args)
    if args.workload == "serve":
        # The server runs dozens of streams at once; CUDA maps streams onto this many
        # hardware queues (default 8), and kernels of streams sharing a queue serialise.
        # Read when the context is created, so it is set before any CUDA call.
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
        return serve_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
