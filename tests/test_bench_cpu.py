"""bench.py's contract where no GPU is needed: the reference arm's JSON line (the keys the
benchmark contract asks for, the CPU reference Rgemm timed on a column slice) and the
shapes of the GEMM arm, square and LU trailing update."""
import json
import os
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
