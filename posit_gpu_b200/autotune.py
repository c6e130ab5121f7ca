"""Autotuner for the batched GEMM tile shapes and the blocked LU / Cholesky panel widths.

Replaces the reference's single OPENCL_GEMM_BLOCKSIZE knob (Rgemm_opencl.cpp:62-66) with
measured choices.  Results never depend on either choice -- tiles do not change the
per-element order of a GEMM, and LU / lower Cholesky in the reference's order are
independent of the block size -- so the tuner is free to pick the fastest.

    python -m posit_gpu_b200.autotune [--out FILE]

writes a JSON table; `load()` returns the table used by default (tuning_b200.json next to
this file, measured on a B200), and `gemm_tile_table()` / `panel_width(n)` read it.
"""
import argparse
import json
import math
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning_b200.json")
BUCKETS = [(4, 32), (33, 64), (65, 512)]  # the size buckets of the tile table
_cache = None


def load(path=None):
    global _cache
    if path is None and _cache is not None:
        return _cache
    p = path or DEFAULT_TABLE
    table = {"gemm_tile_table": None, "panel_width": {}}
    if os.path.exists(p):
        with open(p) as f:
            table.update(json.load(f))
    if path is None:
        _cache = table
    return table


def gemm_tile_table():
    """9 ints for posit_batch_gemm_plan_create, or None for the library default."""
    return load().get("gemm_tile_table")


def panel_width(n, kind="lu"):
    """Tuned nb for an n x n factorization (nearest tuned size at or below n)."""
    pw = load().get("panel_width", {}).get(kind, {})
    best = 256
    for size in sorted(pw, key=int):
        if int(size) <= n:
            best = int(pw[size])
    return best


def _timeit(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return sorted(ts)[len(ts) // 2]


def _rand_posit(numel, gen, dev):
    import torch

    from . import from_double_dev
    x = torch.rand(max(1, numel), dtype=torch.float64, device=dev, generator=gen) * 2 - 1
    return from_double_dev(x)


def tune_gemm_tiles(per_bucket=150, seed=7):
    """Time each tile shape on a sample of GEMMs from each (m, n) size bucket."""
    import torch

    from . import BatchGemmPlan, P32_MINUS_ONE, P32_ONE
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rng = torch.Generator()
    rng.manual_seed(seed)

    def logu(lo, hi):
        u = float(torch.rand(1, generator=rng))
        return int(round(math.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))))

    table, detail = [], {}
    for bi, (mlo, mhi) in enumerate(BUCKETS):
        for bj, (nlo, nhi) in enumerate(BUCKETS):
            probs = []
            for _ in range(per_bucket):
                m, n, k = logu(mlo, mhi), logu(nlo, nhi), logu(4, 512)
                ta = "N" if float(torch.rand(1, generator=rng)) < 0.5 else "T"
                tb = "N" if float(torch.rand(1, generator=rng)) < 0.5 else "T"
                A, B, C = _rand_posit(m * k, gen, dev), _rand_posit(k * n, gen, dev), _rand_posit(m * n, gen, dev)
                lda = m if ta == "N" else k
                ldb = k if tb == "N" else n
                probs.append((ta, tb, m, n, k, P32_MINUS_ONE, A, lda, B, ldb, P32_ONE, C, m))
            times = []
            for cfg in range(3):
                plan = BatchGemmPlan(probs, tile_table=[cfg] * 9)
                times.append(_timeit(plan.launch))
            best = min(range(3), key=lambda c: times[c])
            table.append(best)
            detail[f"m{mlo}-{mhi}_n{nlo}-{nhi}"] = {"ms": times, "best": best}
    return table, detail


def tune_panel_width(sizes=(256, 512, 1024, 2048, 4096, 8192), widths=(16, 24, 32, 48, 64, 128), seed=11):
    """Time the device LU and Cholesky for each panel width at each size."""
    import torch

    from . import Rgetrf_dev, Rpotrf_dev
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    out = {"lu": {}, "chol": {}}
    detail = {}
    for n in sizes:
        A0 = _rand_posit(n * n, gen, dev)
        M = torch.rand(n, n, dtype=torch.float64, device=dev, generator=gen) * 2 - 1
        from . import from_double_dev
        S0 = from_double_dev((M @ M.t() / n + torch.eye(n, dtype=torch.float64, device=dev)).t().contiguous()
                             .reshape(-1))
        ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
        info = torch.zeros(1, dtype=torch.int32, device=dev)
        for kind, src in (("lu", A0), ("chol", S0)):
            times = []
            for nb in widths:
                A = src.clone()

                def run():
                    A.copy_(src)
                    if kind == "lu":
                        Rgetrf_dev(n, n, A, n, ipiv, info, nb=nb)
                    else:
                        Rpotrf_dev("L", n, A, n, info, nb=nb)
                times.append(_timeit(run, reps=2))
            best = widths[min(range(len(widths)), key=lambda i: times[i])]
            out[kind][str(n)] = best
            detail[f"{kind}_{n}"] = {"ms": dict(zip(map(str, widths), times)), "best": best}
    return out, detail


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--per-bucket", type=int, default=150)
    ap.add_argument("--sizes", default="256,512,1024,2048,4096,8192", help="panel widths: matrix sizes")
    args = ap.parse_args()
    import torch
    t0 = time.time()
    tiles, tdet = tune_gemm_tiles(args.per_bucket)
    widths, wdet = tune_panel_width(sizes=tuple(int(x) for x in args.sizes.split(",")))
    res = {"device": torch.cuda.get_device_name(), "gemm_tile_table": tiles, "panel_width": widths,
           "detail": {"gemm_tiles": tdet, "panel_width": wdet}, "seconds": round(time.time() - t0, 1)}
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({"gemm_tile_table": tiles, "panel_width": widths}))


if __name__ == "__main__":
    main()
