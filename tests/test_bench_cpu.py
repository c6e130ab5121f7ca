"""bench.py's contract where no GPU is needed: the reference arm's JSON line (the keys the
benchmark contract asks for, the CPU reference Rgemm timed on a column slice), the shapes
of the GEMM arm, square and LU trailing update, and the multi-rank path: two ranks over
gloo agree on the slowest rank's time, the job's rate counts both replicas, and only rank
0 of the reference arm prints."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _args(*argv):
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_gemm_arm_shapes():
    assert bench.shape(_args()) == (8192, 8192, 8192)
    a = _args("--trailing", "64")
    assert bench.shape(a) == (8128, 8128, 64)
    cfg = bench.config(a)
    assert (cfg["m"], cfg["n"], cfg["k"]) == (8128, 8128, 64)
    assert "trailing update of 8192, b=64" in cfg["workload"]


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "256",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["kind"] in ("reference", "port")


def _rank(rank, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    try:
        t = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")  # rank 1 is the slower one
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out, f"rank{rank}.json"), "w") as fh:
        json.dump({"ms_max": t}, fh)


def test_two_ranks_take_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_rank, args=(port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in (0, 1):
        assert json.load(open(tmp_path / f"rank{r}.json"))["ms_max"] == 20.0
    # whole-job rate: both replicas' work over the slowest rank's time
    assert bench.whole_job_rate(2, 1e9, 3, 20.0) == 2 * 1e9 * 3 / 0.020


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "256",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT,
                       env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""
