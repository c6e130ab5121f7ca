"""Seeded synthetic posit32 operands with the benchmark configurations' shapes and
distributions, generated on the device.

* ``uniform``: entries uniform in [-1, 1] as FP64, converted to posit32 (correctly
  rounded, posit_from_double_dev);
* ``wide``: magnitudes 10^U(-20, 20) with random signs, the wide-dynamic-range variant
  that exercises long regimes.

The benchmark and the parity tests both call :func:`gemm_operands`, so the tests check
the very problem the benchmark times (same seed, same shapes, same bits).
"""
import torch

from . import from_double_dev

GEMM_SEED = 1234


def _fp64(numel, dist, g, dev):
    u = torch.rand(numel, dtype=torch.float64, device=dev, generator=g)
    if dist == "uniform":
        return u * 2.0 - 1.0
    if dist == "wide":
        s = torch.rand(numel, dtype=torch.float64, device=dev, generator=g)
        mag = torch.pow(10.0, u * 40.0 - 20.0)
        return torch.where(s < 0.5, -mag, mag)
    raise ValueError(f"unknown distribution {dist!r}")


def gemm_operands(m, n, k, ta="N", tb="N", seed=GEMM_SEED, device=None, dist="uniform"):
    """A (op(A) is m x k), B (op(B) is k x n) and C (m x n): flat column-major int32
    tensors of posit32 patterns on `device`, with packed leading dimensions.  Returns
    (A, lda, B, ldb, C, ldc).  Generation order is A, B, C from one generator."""
    dev = torch.device(device) if device is not None else torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lda = m if ta in "nN" else k
    ldb = k if tb in "nN" else n
    A = from_double_dev(_fp64(m * k, dist, g, dev))
    B = from_double_dev(_fp64(k * n, dist, g, dev))
    C = from_double_dev(_fp64(m * n, dist, g, dev))
    return A, max(1, lda), B, max(1, ldb), C, max(1, m)
